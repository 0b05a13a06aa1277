"""ctypes binding of the C ABI in include/scdat_b200.h.

This is a thin harness for tests and the benchmark: every call goes straight through the
shared library.  ``load()`` raises when libscdat_b200.so is missing -- there is no fallback.
"""
from __future__ import annotations

import ctypes as C
import weakref
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libscdat_b200.so")

PREC_FP64, PREC_MIXED = 0, 1
PRECOND_JACOBI, PRECOND_MULTIGRID = 0, 1
PUSH_AUTO, PUSH_WALKING, PUSH_STAY_FIRST = 0, 1, 2
DEP_NEAREST, DEP_LINEAR, DEP_GAUSS3 = 0, 1, 2
BC_NONE, BC_ABSORB, BC_PERIODIC = 0, 1, 2
ACTIVE, ABSORBED, ESCAPED = 0, 1, 2
ERR_NOT_CONVERGED = -5


class MeshDesc(C.Structure):
    _fields_ = [("n_nodes", C.c_int64), ("n_tets", C.c_int64), ("node_xyz", C.c_void_p), ("tet_nodes", C.c_void_p),
                ("tet_neighbors", C.c_void_p), ("node_dirichlet", C.c_void_p), ("tet_eps_rel", C.c_void_p)]


class Params(C.Structure):
    _fields_ = [("dt", C.c_double), ("deposit_kernel", C.c_int32), ("deposit_segments", C.c_int32),
                ("adaptive_floor_ratio", C.c_double), ("precision", C.c_int32), ("use_neighbor_lists", C.c_int32),
                ("face_bc", C.c_int32 * 6), ("body_tally", C.c_int32), ("poisson_charge_sign", C.c_int32),
                ("pcg_rtol", C.c_double), ("pcg_max_iter", C.c_int32), ("sort_interval", C.c_int32),
                ("particle_capacity", C.c_int64), ("seed", C.c_uint64)]


class SpeciesC(C.Structure):
    _fields_ = [("charge", C.c_double), ("mass", C.c_double), ("weight", C.c_double), ("electron_like", C.c_int32),
                ("pad", C.c_int32)]


class ElasticC(C.Structure):
    _fields_ = [("target_density", C.c_double), ("sigma_max", C.c_double), ("e_ref_ev", C.c_double),
                ("alpha", C.c_double), ("e_threshold_ev", C.c_double), ("enabled", C.c_int32), ("mode", C.c_int32)]


class BatchTuning(C.Structure):
    _fields_ = [("push_blocks_per_sm", C.c_int32), ("field_blocks_per_sm", C.c_int32), ("use_graph", C.c_int32),
                ("pad", C.c_int32)]


class SurfaceCircuitC(C.Structure):
    _fields_ = [("body_lo", C.c_double * 3), ("body_hi", C.c_double * 3), ("eps_r", C.c_double * 6),
                ("thickness", C.c_double * 6), ("area", C.c_double * 6), ("v0", C.c_double * 6),
                ("shunt_s", C.c_double * 6), ("didv", C.c_double * 6)]


class CurrentSampleC(C.Structure):
    _fields_ = [("surface_potential_v", C.c_double), ("electron_collection_a_per_m2", C.c_double),
                ("ion_collection_a_per_m2", C.c_double), ("emitted_electron_a_per_m2", C.c_double),
                ("net_collection_a_per_m2", C.c_double), ("current_derivative_a_per_m2_per_v", C.c_double),
                ("valid", C.c_int32), ("window_steps", C.c_int32)]


class AdjointRequestC(C.Structure):
    _fields_ = [("steps", C.c_int32), ("checkpoint", C.c_int32), ("g_phi", C.c_void_p), ("g_V", C.c_double * 6),
                ("g_Q", C.c_double * 6), ("bias_nodes", C.c_void_p), ("n_bias_nodes", C.c_int64), ("te_ev", C.c_double)]


class AdjointResultC(C.Structure):
    _fields_ = [("J", C.c_double), ("dJ_dbias", C.c_double), ("dJ_dte", C.c_double), ("dJ_ddelta_max", C.c_double),
                ("flags", C.c_int64)]


class StatsC(C.Structure):
    _fields_ = [("completed_steps", C.c_int64), ("simulation_time", C.c_double), ("total_charge", C.c_double),
                ("total_energy", C.c_double), ("active_particles", C.c_int64), ("stored_particles", C.c_int64),
                ("surface_deposited_charge", C.c_double), ("substeps", C.c_int64), ("lost_events", C.c_int64),
                ("mcc_collisions", C.c_int64), ("last_pcg_iterations", C.c_int32), ("pad", C.c_int32),
                ("last_pcg_relres", C.c_double)]


# every symbol declared in include/scdat_b200.h
EXPORTS = ["scdat_default_params", "scdat_create", "scdat_destroy", "scdat_last_error", "scdat_set_species",
           "scdat_set_particles", "scdat_seed_box_particles", "scdat_kuhn_box_mesh", "scdat_get_particle_count",
           "scdat_get_particles", "scdat_set_potential", "scdat_set_node_potentials", "scdat_set_electric_field",
           "scdat_set_elastic_mcc", "scdat_step", "scdat_push", "scdat_solve_field", "scdat_collide", "scdat_compact",
           "scdat_set_species_sort_interval", "scdat_set_field_preconditioner", "scdat_set_species_push_mode",
           "scdat_get_field_solver_levels",
           "scdat_get_fields", "scdat_get_species_charge", "scdat_get_ledger", "scdat_reset_ledger",
           "scdat_get_statistics", "scdat_version", "scdat_stream", "scdat_set_timing", "scdat_get_timing",
           "scdat_get_sort_timing",
           "scdat_pcg_csr", "scdat_pcg_csr_noalloc", "scdat_set_charge_density", "scdat_set_dt", "scdat_set_seed",
           "scdat_batch_default_tuning", "scdat_batch_create", "scdat_batch_destroy", "scdat_batch_last_error",
           "scdat_batch_step", "scdat_batch_set_tuning", "scdat_batch_get_tuning", "scdat_batch_autotune",
           "scdat_batch_last_step_ms", "scdat_batch_stream", "scdat_batch_kernel_launches",
           "scdat_set_surface_circuit", "scdat_get_surface_state", "scdat_set_secondary_emission",
           "scdat_set_secondary_yield_params",
           "scdat_sample_with_derivative", "scdat_adjoint_window", "scdat_seed_tet_particles",
           "scdat_export_layer_profile_csv", "scdat_export_nodes_csv", "scdat_export_columns_csv"]

_LIB = None


def load():
    """Load the shared library (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m scdat_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.scdat_default_params.argtypes = [C.POINTER(Params)]
    L.scdat_default_params.restype = None
    L.scdat_create.argtypes = [C.POINTER(MeshDesc), C.POINTER(Params), C.POINTER(vp)]
    L.scdat_destroy.argtypes = [vp]
    L.scdat_last_error.argtypes = [vp]
    L.scdat_last_error.restype = C.c_char_p
    L.scdat_set_species.argtypes = [vp, C.c_int32, C.POINTER(SpeciesC)]
    L.scdat_set_charge_density.argtypes = [vp, vp]
    L.scdat_set_dt.argtypes = [vp, C.c_double]
    L.scdat_set_seed.argtypes = [vp, C.c_uint64]
    L.scdat_batch_default_tuning.argtypes = [C.POINTER(BatchTuning)]
    L.scdat_batch_default_tuning.restype = None
    L.scdat_batch_create.argtypes = [C.c_int32, C.POINTER(vp), C.POINTER(vp)]
    L.scdat_batch_destroy.argtypes = [vp]
    L.scdat_batch_last_error.argtypes = [vp]
    L.scdat_batch_last_error.restype = C.c_char_p
    L.scdat_batch_step.argtypes = [vp, C.c_int32]
    L.scdat_batch_set_tuning.argtypes = [vp, C.POINTER(BatchTuning)]
    L.scdat_batch_get_tuning.argtypes = [vp, C.POINTER(BatchTuning)]
    L.scdat_batch_autotune.argtypes = [vp, C.c_int32, C.POINTER(BatchTuning)]
    L.scdat_batch_last_step_ms.argtypes = [vp, C.POINTER(C.c_double)]
    L.scdat_batch_stream.argtypes = [vp, C.POINTER(vp)]
    L.scdat_set_surface_circuit.argtypes = [vp, C.POINTER(SurfaceCircuitC)]
    L.scdat_get_surface_state.argtypes = [vp, vp, vp, vp, vp]
    L.scdat_set_secondary_emission.argtypes = [vp, C.c_int32, C.c_double, C.c_double]
    L.scdat_set_secondary_yield_params.argtypes = [vp, C.c_double, vp]
    L.scdat_seed_tet_particles.argtypes = [vp, C.c_int32, C.c_int64, vp, C.c_int32, C.c_double, vp, C.c_uint64]
    L.scdat_export_layer_profile_csv.argtypes = [vp, C.c_char_p, C.c_int32]
    L.scdat_export_nodes_csv.argtypes = [vp, C.c_char_p]
    L.scdat_export_columns_csv.argtypes = [C.c_char_p, C.c_char_p, C.c_int64, vp, C.c_int32, C.POINTER(C.c_char_p),
                                           C.POINTER(vp)]
    L.scdat_adjoint_window.argtypes = [vp, C.POINTER(AdjointRequestC), C.POINTER(AdjointResultC)]
    L.scdat_sample_with_derivative.argtypes = [C.POINTER(vp), C.c_int64, vp, C.c_int32, C.c_double, C.c_double,
                                               C.c_int32, C.c_double, C.POINTER(CurrentSampleC)]
    L.scdat_batch_kernel_launches.argtypes = [vp, C.POINTER(C.c_int64)]
    L.scdat_set_particles.argtypes = [vp, C.c_int32, C.c_int64, vp, vp, vp, vp]
    L.scdat_seed_box_particles.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_double, vp, vp,
                                           C.c_int32, C.c_double, C.c_uint64]
    L.scdat_kuhn_box_mesh.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_double, vp, vp, C.c_double, C.c_double,
                                      C.POINTER(C.c_int64), C.POINTER(C.c_int64), vp, vp, vp, vp, vp,
                                      C.POINTER(C.c_int64)]
    L.scdat_get_particle_count.argtypes = [vp, C.c_int32, C.POINTER(C.c_int64)]
    L.scdat_get_particles.argtypes = [vp, C.c_int32, C.c_int64, vp, vp, vp, vp, vp, C.POINTER(C.c_int64)]
    L.scdat_set_potential.argtypes = [vp, vp]
    L.scdat_set_node_potentials.argtypes = [vp, C.c_int64, vp, vp]
    L.scdat_set_electric_field.argtypes = [vp, vp]
    L.scdat_set_elastic_mcc.argtypes = [vp, C.c_int32, C.POINTER(ElasticC)]
    for f in ("scdat_push", "scdat_solve_field", "scdat_collide", "scdat_compact", "scdat_reset_ledger"):
        getattr(L, f).argtypes = [vp]
    L.scdat_step.argtypes = [vp, C.c_int32]
    L.scdat_set_species_sort_interval.argtypes = [vp, C.c_int32, C.c_int32]
    L.scdat_set_field_preconditioner.argtypes = [vp, C.c_int32]
    L.scdat_set_species_push_mode.argtypes = [vp, C.c_int32, C.c_int32]
    L.scdat_get_field_solver_levels.argtypes = [vp, C.c_int32, vp, vp, vp, vp]
    L.scdat_get_fields.argtypes = [vp, vp, vp, vp]
    L.scdat_get_species_charge.argtypes = [vp, C.c_int32, vp]
    L.scdat_get_ledger.argtypes = [vp, vp]
    L.scdat_get_statistics.argtypes = [vp, C.POINTER(StatsC)]
    L.scdat_stream.argtypes = [vp]
    L.scdat_stream.restype = vp
    L.scdat_set_timing.argtypes = [vp, C.c_int32]
    L.scdat_get_timing.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                   C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.scdat_get_sort_timing.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_int64)]
    L.scdat_pcg_csr.argtypes = [C.c_int32, vp, vp, vp, vp, vp, vp, C.c_double, C.c_int32, vp,
                                C.POINTER(C.c_int32), C.POINTER(C.c_double)]
    L.scdat_pcg_csr_noalloc.argtypes = L.scdat_pcg_csr.argtypes
    L.scdat_version.argtypes = []
    L.scdat_version.restype = C.c_char_p
    _LIB = L
    return L


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def kuhn_box_mesh(n, h, body=None, bias=0.0, wall=0.0):
    """Mesh arrays of the 6-tet Kuhn box built by the library (scdat_kuhn_box_mesh)."""
    L = load()
    nx, ny, nz = n
    lo = hi = None
    if body is not None:
        lo = np.array([body[0][0], body[1][0], body[2][0]], np.int32)
        hi = np.array([body[0][1], body[1][1], body[2][1]], np.int32)
    N = C.c_int64()
    T = C.c_int64()
    nc = C.c_int64()
    rc = L.scdat_kuhn_box_mesh(nx, ny, nz, h, _p(lo), _p(hi), bias, wall, C.byref(N), C.byref(T), None, None, None,
                               None, None, C.byref(nc))
    assert rc == 0
    xyz = np.zeros((N.value, 3))
    tet = np.zeros((T.value, 4), np.int32)
    dirichlet = np.zeros(N.value, np.uint8)
    phi = np.zeros(N.value)
    hexes = np.zeros((nc.value, 3), np.int32)
    rc = L.scdat_kuhn_box_mesh(nx, ny, nz, h, _p(lo), _p(hi), bias, wall, C.byref(N), C.byref(T), _p(xyz), _p(tet),
                               _p(dirichlet), _p(phi), _p(hexes), C.byref(nc))
    assert rc == 0
    return dict(xyz=xyz, tet=tet, dirichlet=dirichlet, phi=phi, hex_ijk=hexes)


class ScdatError(RuntimeError):
    def __init__(self, rc, msg):
        super().__init__(f"scdat error {rc}: {msg}")
        self.rc = rc


class Domain:
    """One device context: mesh, fields, species and their particles."""

    def __init__(self, xyz, tet, dirichlet, dt, *, nbr=None, eps_rel=None, precision=PREC_FP64, face_bc=(0,) * 6,
                 deposit_kernel=DEP_LINEAR, deposit_segments=10, use_neighbor_lists=True, pcg_rtol=1e-8,
                 pcg_max_iter=5000, sort_interval=0, charge_sign=-1, body_tally=True, seed=0x5CDA7B200,
                 floor_ratio=0.001):
        self.L = load()
        self.xyz = np.ascontiguousarray(xyz, np.float64)
        self.tet = np.ascontiguousarray(tet, np.int32)
        self.dirichlet = np.ascontiguousarray(dirichlet, np.uint8)
        self.nbr = None if nbr is None else np.ascontiguousarray(nbr, np.int32)
        self.eps_rel = None if eps_rel is None else np.ascontiguousarray(eps_rel, np.float64)
        self.N = self.xyz.shape[0]
        self.T = self.tet.shape[0]
        md = MeshDesc(self.N, self.T, _p(self.xyz), _p(self.tet), _p(self.nbr), _p(self.dirichlet), _p(self.eps_rel))
        prm = Params()
        self.L.scdat_default_params(C.byref(prm))
        prm.dt = dt
        prm.precision = precision
        for f in range(6):
            prm.face_bc[f] = face_bc[f]
        prm.deposit_kernel = deposit_kernel
        prm.deposit_segments = deposit_segments
        prm.use_neighbor_lists = 1 if use_neighbor_lists else 0
        prm.pcg_rtol = pcg_rtol
        prm.pcg_max_iter = pcg_max_iter
        prm.sort_interval = sort_interval
        prm.poisson_charge_sign = charge_sign
        prm.body_tally = 1 if body_tally else 0
        prm.seed = seed
        prm.adaptive_floor_ratio = floor_ratio
        self.params = prm
        h = C.c_void_p()
        rc = self.L.scdat_create(C.byref(md), C.byref(prm), C.byref(h))
        if rc != 0:
            raise ScdatError(rc, "scdat_create: " + self.L.scdat_last_error(None).decode())
        self.h = h
        self.nspecies = 0
        self._batches = weakref.WeakSet()  # Batches holding this Domain

    def _ck(self, rc):
        if rc != 0:
            raise ScdatError(rc, self.L.scdat_last_error(self.h).decode())
        return rc

    def close(self):
        # A Batch's graph points into this Domain's buffers, and the library refuses to destroy a
        # context a batch still holds: close those batches first.  This also holds when the
        # garbage collector finalises a cycle holding both in an arbitrary order.
        for b in list(getattr(self, "_batches", ())):
            b.close()
        if getattr(self, "h", None):
            self._ck(self.L.scdat_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def rows(self):
        """Interior (non-Dirichlet) nodes: the rows of the reduced Poisson system."""
        return int(np.count_nonzero(self.dirichlet == 0))

    def set_species(self, species):
        arr = (SpeciesC * len(species))(*[SpeciesC(s.q, s.m, s.w, 1 if s.q < 0 else 0, 0) for s in species])
        self._ck(self.L.scdat_set_species(self.h, len(species), arr))
        self.nspecies = len(species)

    def set_particles(self, s, x, v, tet=None, ids=None):
        x = np.ascontiguousarray(x, np.float64)
        v = np.ascontiguousarray(v, np.float64)
        t = None if tet is None else np.ascontiguousarray(tet, np.int32)
        i = None if ids is None else np.ascontiguousarray(ids, np.uint32)
        self._ck(self.L.scdat_set_particles(self.h, s, x.shape[0], _p(x), _p(v), _p(t), _p(i)))

    def seed_box(self, s, n, h, body, ppc, temp_ev, seed):
        lo = hi = None
        if body is not None:
            lo = np.array([body[0][0], body[1][0], body[2][0]], np.int32)
            hi = np.array([body[0][1], body[1][1], body[2][1]], np.int32)
        self._ck(self.L.scdat_seed_box_particles(self.h, s, n[0], n[1], n[2], h, _p(lo), _p(hi), ppc, temp_ev, seed))

    def count(self, s):
        n = C.c_int64()
        self._ck(self.L.scdat_get_particle_count(self.h, s, C.byref(n)))
        return n.value

    def get_particles(self, s):
        n = self.count(s)
        x = np.zeros((n, 3))
        v = np.zeros((n, 3))
        t = np.zeros(n, np.int32)
        st = np.zeros(n, np.uint8)
        ids = np.zeros(n, np.uint32)
        nn = C.c_int64()
        self._ck(self.L.scdat_get_particles(self.h, s, n, _p(x), _p(v), _p(t), _p(st), _p(ids), C.byref(nn)))
        return dict(x=x, v=v, tet=t, status=st, id=ids)

    def set_potential(self, phi):
        phi = np.ascontiguousarray(phi, np.float64)
        self._ck(self.L.scdat_set_potential(self.h, _p(phi)))

    def set_node_potentials(self, nodes, values):
        nodes = np.ascontiguousarray(nodes, np.int64)
        values = np.ascontiguousarray(values, np.float64)
        self._ck(self.L.scdat_set_node_potentials(self.h, nodes.shape[0], _p(nodes), _p(values)))

    def set_electric_field(self, E):
        E = np.ascontiguousarray(E, np.float64)
        self._ck(self.L.scdat_set_electric_field(self.h, _p(E)))

    def set_charge_density(self, rho):
        rho = np.ascontiguousarray(rho, np.float64)
        self._ck(self.L.scdat_set_charge_density(self.h, _p(rho)))

    def set_dt(self, dt):
        self._ck(self.L.scdat_set_dt(self.h, float(dt)))

    def set_seed(self, seed):
        self._ck(self.L.scdat_set_seed(self.h, int(seed)))

    def seed_tets(self, s, n_per_tet, temp_ev, seed, tets=None, drift=None):
        """scdat_seed_tet_particles (all tets when `tets` is None)."""
        t = None if tets is None else np.ascontiguousarray(tets, np.int32)
        d = None if drift is None else np.ascontiguousarray(drift, np.float64)
        self._ck(self.L.scdat_seed_tet_particles(self.h, s, 0 if t is None else t.shape[0], _p(t), int(n_per_tet),
                                                 float(temp_ev), _p(d), int(seed)))

    def export_layer_profile(self, path, n_layers):
        self._ck(self.L.scdat_export_layer_profile_csv(self.h, str(path).encode(), int(n_layers)))

    def export_nodes(self, path):
        self._ck(self.L.scdat_export_nodes_csv(self.h, str(path).encode()))

    def set_surface_circuit(self, body_lo, body_hi, eps_r=3.0, thickness=1e-3, v0=0.0, shunt=0.0, didv=0.0,
                            area=0.0):
        """Faces XMin..ZMax of the body box as floating dielectric patches (scalars apply to all)."""
        sc = SurfaceCircuitC()
        for a in range(3):
            sc.body_lo[a] = body_lo[a]
            sc.body_hi[a] = body_hi[a]
        for name, val in (("eps_r", eps_r), ("thickness", thickness), ("v0", v0), ("shunt_s", shunt),
                          ("didv", didv), ("area", area)):
            arr = np.broadcast_to(np.asarray(val, np.float64), (6,))
            for f in range(6):
                getattr(sc, name)[f] = float(arr[f])
        self._ck(self.L.scdat_set_surface_circuit(self.h, C.byref(sc)))

    def set_secondary_emission(self, model, delta_max=2.0, e_max_ev=300.0):
        """model: 0 off, 1 Sternglass, 2 Whipple, 3 Sims, 4 Katz (the reference's legacy forms)."""
        self._ck(self.L.scdat_set_secondary_emission(self.h, int(model), float(delta_max), float(e_max_ev)))

    def set_secondary_yield_params(self, sims_exponent_n=1.6, katz=None):
        """Sims exponent and Katz range coefficients (r1, n1, r2, n2; None: the defaults)."""
        k = None if katz is None else np.ascontiguousarray(katz, np.float64)
        assert k is None or k.shape == (4,)
        self._ck(self.L.scdat_set_secondary_yield_params(self.h, float(sims_exponent_n), _p(k)))

    def surface_state(self):
        V, Q, I = np.zeros(6), np.zeros(6), np.zeros(6)
        n = np.zeros(6, np.int64)
        self._ck(self.L.scdat_get_surface_state(self.h, _p(V), _p(Q), _p(I), _p(n)))
        return dict(V=V, Q=Q, I=I, counts=n)

    def adjoint_window(self, steps, checkpoint=10, g_phi=None, g_V=(0.0,) * 6, g_Q=(0.0,) * 6, bias_nodes=None,
                       te_ev=0.0):
        """scdat_adjoint_window: J and dJ/d(bias, Te, delta_max) over `steps` FP64 steps."""
        rq = AdjointRequestC()
        rq.steps, rq.checkpoint = int(steps), int(checkpoint)
        gp = None if g_phi is None else np.ascontiguousarray(g_phi, np.float64)
        bn = None if bias_nodes is None else np.ascontiguousarray(bias_nodes, np.int64)
        rq.g_phi = None if gp is None else gp.ctypes.data
        for f in range(6):
            rq.g_V[f] = float(g_V[f])
            rq.g_Q[f] = float(g_Q[f])
        rq.bias_nodes = None if bn is None else bn.ctypes.data
        rq.n_bias_nodes = 0 if bn is None else bn.shape[0]
        rq.te_ev = float(te_ev)
        res = AdjointResultC()
        self._ck(self.L.scdat_adjoint_window(self.h, C.byref(rq), C.byref(res)))
        return dict(J=res.J, dbias=res.dJ_dbias, dte=res.dJ_dte, ddelta=res.dJ_ddelta_max, flags=res.flags)

    def set_elastic(self, s, n_target, sigma, mode=0, alpha=0.0, e_ref=1.0, e_th=0.0, enabled=True):
        proc = ElasticC(n_target, sigma, e_ref, alpha, e_th, 1 if enabled else 0, mode)
        self._ck(self.L.scdat_set_elastic_mcc(self.h, s, C.byref(proc)))

    def push(self):
        self._ck(self.L.scdat_push(self.h))

    def solve_field(self, allow_not_converged=False):
        rc = self.L.scdat_solve_field(self.h)
        if rc == ERR_NOT_CONVERGED and allow_not_converged:
            return rc
        return self._ck(rc)

    def collide(self):
        self._ck(self.L.scdat_collide(self.h))

    def compact(self):
        self._ck(self.L.scdat_compact(self.h))

    def set_species_sort_interval(self, species, interval):
        """scdat_set_species_sort_interval: re-sort this species every `interval` steps."""
        self._ck(self.L.scdat_set_species_sort_interval(self.h, int(species), int(interval)))

    def set_push_mode(self, species, mode):
        """scdat_set_species_push_mode: PUSH_AUTO, PUSH_WALKING or PUSH_STAY_FIRST."""
        self._ck(self.L.scdat_set_species_push_mode(self.h, int(species), int(mode)))

    def solver_levels(self):
        """scdat_get_field_solver_levels: [(rows, operator nonzeros, prolongation nonzeros)]."""
        nl = C.c_int32()
        self._ck(self.L.scdat_get_field_solver_levels(self.h, 0, C.byref(nl), None, None, None))
        r, z, t = (np.zeros(nl.value, np.int64) for _ in range(3))
        self._ck(self.L.scdat_get_field_solver_levels(self.h, nl.value, C.byref(nl), _p(r), _p(z), _p(t)))
        return [(int(a), int(b), int(c)) for a, b, c in zip(r, z, t)]

    def set_preconditioner(self, kind):
        """scdat_set_field_preconditioner: PRECOND_JACOBI (default) or PRECOND_MULTIGRID."""
        self._ck(self.L.scdat_set_field_preconditioner(self.h, int(kind)))

    def rows(self):
        """Interior (non-Dirichlet) nodes: the rows of the reduced Poisson system."""
        return int(np.count_nonzero(self.dirichlet == 0))

    def step(self, n=1):
        self._ck(self.L.scdat_step(self.h, n))

    def fields(self):
        rho = np.zeros(self.N)
        phi = np.zeros(self.N)
        E = np.zeros((self.N, 3))
        self._ck(self.L.scdat_get_fields(self.h, _p(rho), _p(phi), _p(E)))
        return rho, phi, E

    def species_charge(self, s):
        r = np.zeros(self.N)
        self._ck(self.L.scdat_get_species_charge(self.h, s, _p(r)))
        return r

    def ledger(self):
        led = np.zeros((7, 8))
        self._ck(self.L.scdat_get_ledger(self.h, _p(led)))
        return led

    def reset_ledger(self):
        self._ck(self.L.scdat_reset_ledger(self.h))

    def stream(self):
        return self.L.scdat_stream(self.h)

    def set_timing(self, on=True):
        self._ck(self.L.scdat_set_timing(self.h, 1 if on else 0))

    def timing(self):
        pm, fm = C.c_double(), C.c_double()
        pl, pp, fs, kl = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        self._ck(self.L.scdat_get_timing(self.h, C.byref(pm), C.byref(pl), C.byref(pp), C.byref(fm), C.byref(fs),
                                         C.byref(kl)))
        sm, sn = C.c_double(), C.c_int64()
        self._ck(self.L.scdat_get_sort_timing(self.h, C.byref(sm), C.byref(sn)))
        return dict(push_ms=pm.value, push_launches=pl.value, push_particles=pp.value, field_ms=fm.value,
                    field_solves=fs.value, kernel_launches=kl.value, sort_ms=sm.value, sorts=sn.value)

    def stats(self):
        st = StatsC()
        self._ck(self.L.scdat_get_statistics(self.h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in StatsC._fields_ if k != "pad"}


class Batch:
    """scdat_batch: independent mixed-precision Domains stepped together (one CUDA-graph launch
    per step).  The Domains stay usable for queries; step them only through the batch."""

    def __init__(self, domains, use_graph=True, push_blocks_per_sm=None, field_blocks_per_sm=None):
        self.L = load()
        self.domains = list(domains)
        arr = (C.c_void_p * len(self.domains))(*[d.h for d in self.domains])
        h = C.c_void_p()
        rc = self.L.scdat_batch_create(len(self.domains), arr, C.byref(h))
        self.h = h
        if rc != 0:
            msg = self.L.scdat_batch_last_error(h).decode() if h.value else "batch create failed"
            if h.value:
                self.L.scdat_batch_destroy(h)
            self.h = None
            raise ScdatError(rc, msg)
        for d in self.domains:
            d._batches.add(self)
        t = self.tuning()
        t.use_graph = 1 if use_graph else 0
        if push_blocks_per_sm:
            t.push_blocks_per_sm = push_blocks_per_sm
        if field_blocks_per_sm:
            t.field_blocks_per_sm = field_blocks_per_sm
        self.set_tuning(t)

    def _ck(self, rc):
        if rc != 0:
            raise ScdatError(rc, self.L.scdat_batch_last_error(self.h).decode())
        return rc

    def tuning(self):
        t = BatchTuning()
        self._ck(self.L.scdat_batch_get_tuning(self.h, C.byref(t)))
        return t

    def set_tuning(self, t):
        self._ck(self.L.scdat_batch_set_tuning(self.h, C.byref(t)))

    def step(self, n=1):
        self._ck(self.L.scdat_batch_step(self.h, int(n)))

    def autotune(self, steps_each=1):
        t = BatchTuning()
        self._ck(self.L.scdat_batch_autotune(self.h, int(steps_each), C.byref(t)))
        return dict(push_blocks_per_sm=t.push_blocks_per_sm, field_blocks_per_sm=t.field_blocks_per_sm,
                    use_graph=t.use_graph)

    def stream(self):
        v = C.c_void_p()
        self._ck(self.L.scdat_batch_stream(self.h, C.byref(v)))
        return v.value

    def kernel_launches(self):
        v = C.c_int64()
        self._ck(self.L.scdat_batch_kernel_launches(self.h, C.byref(v)))
        return v.value

    def last_step_ms(self):
        v = C.c_double()
        self._ck(self.L.scdat_batch_last_step_ms(self.h, C.byref(v)))
        return v.value

    def close(self):
        if getattr(self, "h", None):
            self.L.scdat_batch_destroy(self.h)
            self.h = None
            for d in getattr(self, "domains", ()):
                d._batches.discard(self)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


LEDGER_BODY = 6  # ledger rows 0..5 are the domain faces XMin..ZMax


def export_columns_csv(path, axis_name, axis, series):
    """scdat_export_columns_csv (CSVExporter::exportDataSet) of {name: values} over the axis."""
    L = load()
    names = list(series)
    vals = [np.ascontiguousarray(series[k], np.float64) for k in names]
    a = np.ascontiguousarray(axis, np.float64)
    assert all(v.shape == a.shape for v in vals)
    cn = (C.c_char_p * max(1, len(names)))(*[k.encode() for k in names])
    cv = (C.c_void_p * max(1, len(names)))(*[v.ctypes.data for v in vals])
    rc = L.scdat_export_columns_csv(str(path).encode(), axis_name.encode(), a.shape[0], _p(a), len(names), cn, cv)
    if rc != 0:
        raise ScdatError(rc, "scdat_export_columns_csv failed")


def sample_with_derivative(domains, surface_nodes, surface_potential_v, probe_delta_v, window_steps, area_m2,
                           ledger_row=LEDGER_BODY):
    """scdat_sample_with_derivative over three Domains holding the same scenario; the collected
    charge is that of `ledger_row` (a face 0..5, or the body box)."""
    L = load()
    arr = (C.c_void_p * 3)(*[d.h for d in domains])
    nodes = np.ascontiguousarray(surface_nodes, np.int64)
    out = CurrentSampleC()
    rc = L.scdat_sample_with_derivative(arr, nodes.shape[0], _p(nodes), int(ledger_row), float(surface_potential_v),
                                        float(probe_delta_v), int(window_steps), float(area_m2), C.byref(out))
    if rc != 0:
        raise ScdatError(rc, L.scdat_last_error(domains[1].h).decode())
    return {k: getattr(out, k) for k, _ in CurrentSampleC._fields_}

