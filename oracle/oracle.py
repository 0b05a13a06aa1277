"""Python access to the parity checkers (TEST INFRASTRUCTURE ONLY).

* ``Oracle``   -- ctypes wrapper of liboracle.so, the C restatement in scdat_oracle.c.
* ``Reference`` -- ctypes wrapper of _ref/libscdat_ref.so, the reference's own classes
  compiled from its sources (present only where the reference tree was available at build
  time).
* numpy builders for the benchmark geometry: a box of n^3 hex cells, each split into the
  6 Kuhn tetrahedra, with an optional hole for a conducting body, and seeded particles.

Only tests/, the smoke check and the benchmark's CPU-baseline leg import this module.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libscdat_ref.so")
REF_OMP_SO = os.path.join(HERE, "_ref", "libscdat_ref_omp.so")

QE = 1.602176634e-19          # Constants.h:46
ME = 9.1093837015e-31         # Constants.h:47
MP = 1.67262192369e-27        # Constants.h:48
EPS0 = 8.8541878128e-12       # PoissonSolver.cpp:18

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")


def build_oracle() -> None:
    """Compile liboracle.so if it is missing (gcc only; no reference tree needed)."""
    if not os.path.exists(ORACLE_SO):
        subprocess.check_call(["make", "-C", HERE, "oracle"], stdout=subprocess.DEVNULL)


def _nullable(arr, dtype):
    if arr is None:
        return None
    return np.ascontiguousarray(arr, dtype=dtype).ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------------------------------
# Mesh and particle builders
# ---------------------------------------------------------------------------------------
KUHN_PERMS = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))


@dataclass
class BoxMesh:
    n: tuple
    h: float
    xyz: np.ndarray          # [N,3] f64
    tet: np.ndarray          # [T,4] i32
    nbr: np.ndarray          # [T,4] i32, neighbour across the face opposite vertex f, -1 none
    dirichlet: np.ndarray    # [N] u8
    phi_bc: np.ndarray       # [N] f64 Dirichlet values (0 elsewhere)
    hex_ijk: np.ndarray      # [C,3] i32 meshed hex cells (compact order)
    body: tuple | None = None

    @property
    def N(self):
        return self.xyz.shape[0]

    @property
    def T(self):
        return self.tet.shape[0]


def face_neighbors(tet: np.ndarray) -> np.ndarray:
    """Neighbour across the face opposite each vertex (-1 on the boundary)."""
    T = tet.shape[0]
    nbr = np.full((T, 4), -1, dtype=np.int32)
    faces = []
    for f in range(4):
        others = np.delete(tet, f, axis=1)
        faces.append(np.sort(others, axis=1))
    F = np.concatenate(faces, axis=0).astype(np.int64)
    owner = np.concatenate([np.arange(T)] * 4)
    slot = np.repeat(np.arange(4), T)
    M = int(tet.max()) + 1 if T else 1
    key = (F[:, 0] * M + F[:, 1]) * M + F[:, 2]
    order = np.argsort(key, kind="stable")
    ks = key[order]
    same = np.nonzero(ks[1:] == ks[:-1])[0]
    a, b = order[same], order[same + 1]
    nbr[owner[a], slot[a]] = owner[b]
    nbr[owner[b], slot[b]] = owner[a]
    return nbr


def kuhn_box(n, h: float, body=None, bias: float = 0.0, wall: float = 0.0) -> BoxMesh:
    """n = (nx, ny, nz) hex cells of edge h from the origin, 6 Kuhn tets per hex.

    body = ((i0,i1),(j0,j1),(k0,k1)) half-open hex index ranges left unmeshed (a conducting
    body); its nodes are Dirichlet at ``bias``.  Outer-face nodes are Dirichlet at ``wall``.
    """
    nx, ny, nz = n
    I, J, K = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    # node id = i + (nx+1)*(j + (ny+1)*k)
    ii = I.transpose(2, 1, 0).ravel()
    jj = J.transpose(2, 1, 0).ravel()
    kk = K.transpose(2, 1, 0).ravel()
    xyz = np.stack([ii * h, jj * h, kk * h], axis=1).astype(np.float64)
    hi, hj, hk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    hex_ijk = np.stack([hi.transpose(2, 1, 0).ravel(), hj.transpose(2, 1, 0).ravel(),
                        hk.transpose(2, 1, 0).ravel()], axis=1).astype(np.int32)
    inb = np.zeros(len(hex_ijk), dtype=bool)
    if body is not None:
        (i0, i1), (j0, j1), (k0, k1) = body
        inb = ((hex_ijk[:, 0] >= i0) & (hex_ijk[:, 0] < i1) & (hex_ijk[:, 1] >= j0) & (hex_ijk[:, 1] < j1)
               & (hex_ijk[:, 2] >= k0) & (hex_ijk[:, 2] < k1))
    hex_ijk = hex_ijk[~inb]

    def nid(i, j, k):
        return i + (nx + 1) * (j + (ny + 1) * k)

    tets = np.empty((len(hex_ijk), 6, 4), dtype=np.int64)
    base = hex_ijk.astype(np.int64)
    for p, perm in enumerate(KUHN_PERMS):
        c = np.zeros((len(base), 3), dtype=np.int64)
        verts = [c.copy()]
        c[:, perm[0]] += 1
        verts.append(c.copy())
        c[:, perm[1]] += 1
        verts.append(c.copy())
        c[:, perm[2]] += 1
        verts.append(c.copy())
        for v_i, off in enumerate(verts):
            q = base + off
            tets[:, p, v_i] = nid(q[:, 0], q[:, 1], q[:, 2])
    tet = tets.reshape(-1, 4).astype(np.int32)
    nbr = face_neighbors(tet)
    N = xyz.shape[0]
    dirichlet = np.zeros(N, dtype=np.uint8)
    phi_bc = np.zeros(N, dtype=np.float64)
    outer = (ii == 0) | (ii == nx) | (jj == 0) | (jj == ny) | (kk == 0) | (kk == nz)
    dirichlet[outer] = 1
    phi_bc[outer] = wall
    if body is not None:
        (i0, i1), (j0, j1), (k0, k1) = body
        inbody = (ii >= i0) & (ii <= i1) & (jj >= j0) & (jj <= j1) & (kk >= k0) & (kk <= k1)
        dirichlet[inbody] = 1
        phi_bc[inbody] = bias
    return BoxMesh(n=(nx, ny, nz), h=h, xyz=xyz, tet=tet, nbr=nbr, dirichlet=dirichlet, phi_bc=phi_bc,
                   hex_ijk=hex_ijk, body=body)


def philox4x32_10(ctr, key):
    """Vectorised Philox4x32-10 (Salmon et al., SC'11); ctr [M,4] u32, key [M,2] u32."""
    c = [ctr[:, i].astype(np.uint64) for i in range(4)]
    k0 = key[:, 0].astype(np.uint64)
    k1 = key[:, 1].astype(np.uint64)
    m32 = np.uint64(0xFFFFFFFF)
    for r in range(10):
        if r:
            k0 = (k0 + np.uint64(0x9E3779B9)) & m32
            k1 = (k1 + np.uint64(0xBB67AE85)) & m32
        p0 = np.uint64(0xD2511F53) * c[0]
        p1 = np.uint64(0xCD9E8D57) * c[2]
        n0 = (p1 >> np.uint64(32)) ^ c[1] ^ k0
        n1 = p1 & m32
        n2 = (p0 >> np.uint64(32)) ^ c[3] ^ k1
        n3 = p0 & m32
        c = [n0, n1, n2, n3]
    return np.stack(c, axis=1).astype(np.uint32)


def uniforms2(seed: int, ids: np.ndarray, step: int, purpose: int) -> np.ndarray:
    """Two (0,1) uniforms per id, same convention as the C oracle and the CUDA kernels."""
    ids = np.asarray(ids, dtype=np.uint64)
    ctr = np.stack([ids & np.uint64(0xFFFFFFFF), ids >> np.uint64(32),
                    np.full_like(ids, step), np.full_like(ids, purpose)], axis=1).astype(np.uint32)
    key = np.tile(np.array([seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF], dtype=np.uint32), (len(ids), 1))
    o = philox4x32_10(ctr, key).astype(np.uint64)
    out = np.empty((len(ids), 2))
    for k in range(2):
        m = ((o[:, 2 * k] << np.uint64(21)) ^ (o[:, 2 * k + 1] >> np.uint64(11))) & np.uint64((1 << 53) - 1)
        out[:, k] = (m.astype(np.float64) + 0.5) * (1.0 / 9007199254740992.0)
    return out


@dataclass
class Species:
    q: float
    m: float
    w: float
    kind: int        # 0 electron-like, 1 H+ ion
    temp_ev: float


def plasma_species(density: float, te_ev: float, ti_ev: float, h: float, ppc: int):
    """Electrons and H+ with macro weight n*h^3/ppc (ParticleDefinitions.cpp:374-392)."""
    w = density * h ** 3 / ppc
    return [Species(-QE, ME, w, 0, te_ev), Species(QE, MP, w, 1, ti_ev)]


def seed_particles(mesh: BoxMesh, species, ppc: int, seed: int):
    """ppc particles per species in every meshed hex, uniform in the hex, Maxwellian.

    Particle id = (cell * S + s) * ppc + k, so arrays are cell-sorted.  Returns dict with
    x [P,3], v [P,3], species [P] i32, tet [P] i32 (the Kuhn tet holding the point), id [P].
    """
    Cn = len(mesh.hex_ijk)
    S = len(species)
    P = Cn * S * ppc
    ids = np.arange(P, dtype=np.int64)
    cell = ids // (S * ppc)
    sp = (ids // ppc) % S
    u01 = uniforms2(seed, ids, 0, 0)
    u2x = uniforms2(seed, ids, 0, 1)
    loc = np.stack([u01[:, 0], u01[:, 1], u2x[:, 0]], axis=1)
    ijk = mesh.hex_ijk[cell].astype(np.float64)
    x = (ijk + loc) * mesh.h
    # Kuhn tet: permutation sorting local coordinates in descending order
    order = np.argsort(-loc, axis=1, kind="stable")
    perm_index = {p: i for i, p in enumerate(KUHN_PERMS)}
    pidx = np.array([perm_index[tuple(r)] for r in order], dtype=np.int32)
    tet = (cell * 6 + pidx).astype(np.int32)
    g1 = uniforms2(seed, ids, 0, 4)
    g2 = uniforms2(seed, ids, 0, 5)
    r1 = np.sqrt(-2.0 * np.log(g1[:, 0]))
    r2 = np.sqrt(-2.0 * np.log(g2[:, 0]))
    nrm = np.stack([r1 * np.cos(2 * np.pi * g1[:, 1]), r1 * np.sin(2 * np.pi * g1[:, 1]),
                    r2 * np.cos(2 * np.pi * g2[:, 1])], axis=1)
    sig = np.array([np.sqrt(s.temp_ev * QE / s.m) for s in species])[sp]
    v = nrm * sig[:, None]
    return dict(x=np.ascontiguousarray(x), v=np.ascontiguousarray(v), species=sp.astype(np.int32),
                tet=tet, id=ids)


# ---------------------------------------------------------------------------------------
# C oracle
# ---------------------------------------------------------------------------------------
class PushParams(C.Structure):
    _fields_ = [("dt", C.c_double), ("floor_ratio", C.c_double), ("nseg", C.c_int32),
                ("dep_kernel", C.c_int32), ("deposit", C.c_int32), ("pad", C.c_int32)]


class PushStats(C.Structure):
    _fields_ = [("substeps", C.c_int64), ("lost", C.c_int64), ("max_iter_hit", C.c_int64), ("pad", C.c_int64)]


class BcParams(C.Structure):
    _fields_ = [("bmin", C.c_double * 3), ("bmax", C.c_double * 3), ("face_bc", C.c_int32 * 6),
                ("period", C.c_double * 3), ("body_tally", C.c_int32), ("pad", C.c_int32)]


class Elastic(C.Structure):
    _fields_ = [("n_target", C.c_double), ("sigma_max", C.c_double), ("e_ref", C.c_double),
                ("alpha", C.c_double), ("e_threshold", C.c_double), ("enabled", C.c_int32), ("pad", C.c_int32)]


BC_NONE, BC_ABSORB, BC_PERIODIC = 0, 1, 2
ACTIVE, ABSORBED, ESCAPED = 0, 1, 2


class Oracle:
    """fast_locate: replace the reference's linear scan over all tets (the last step of
    locateParticle) by the oracle's exact stand-in, a bin grid listing every tet that can hold
    a point in ascending id order (scdat_oracle.c, orc_grid_create), so that meshes of 10^5
    tets and more finish in seconds.  Both give the same tet for every point (tested)."""

    def __init__(self, fast_locate: bool = False):
        build_oracle()
        L = C.CDLL(ORACLE_SO)
        self.L = L
        self.fast_locate = fast_locate
        self._grids = {}
        L.orc_grid_create.argtypes = [_dp, _i32p, C.c_int64]
        L.orc_grid_create.restype = C.c_void_p
        L.orc_grid_destroy.argtypes = [C.c_void_p]
        L.orc_grid_use.argtypes = [C.c_void_p]
        L.orc_philox4x32_10.argtypes = [_u32p, _u32p, _u32p]
        L.orc_barycentric.argtypes = [_dp, _i32p, C.c_int64, _dp, _dp]
        L.orc_barycentric.restype = C.c_int
        L.orc_locate_point.argtypes = [_dp, _i32p, C.c_void_p, C.c_int64, _dp, C.c_int64]
        L.orc_locate_point.restype = C.c_int64
        L.orc_push.argtypes = [C.c_int64, _dp, C.c_int64, _i32p, C.c_void_p, _dp, C.c_int64, _dp, _dp, _i32p,
                               _i32p, _u8p, _u8p, _dp, _dp, _dp, C.POINTER(PushParams), _dp,
                               C.POINTER(PushStats)]
        L.orc_boundary.argtypes = [C.c_int64, _dp, _i32p, C.c_void_p, C.c_int64, _dp, _dp, _i32p, _i32p, _u8p,
                                   _u8p, _dp, _dp, _dp, C.POINTER(BcParams), _dp, _dp]
        L.orc_assemble.argtypes = [C.c_int64, _dp, C.c_int64, _i32p, C.c_void_p, _i64p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.POINTER(C.c_int64)]
        L.orc_poisson_cg.argtypes = [C.c_int64, _i64p, _i32p, _dp, _dp, _dp, _u8p, _dp, C.c_double, _dp,
                                     C.c_double, C.c_int, C.POINTER(C.c_double)]
        L.orc_poisson_cg.restype = C.c_int
        L.orc_lsq_efield.argtypes = [C.c_int64, _dp, _i64p, _i32p, _dp, C.c_double, _dp]
        L.orc_mcc.argtypes = [C.c_int64, _dp, _i32p, _u8p, _i64p, _dp, C.POINTER(Elastic), C.c_double,
                              C.c_uint64, C.c_uint32, C.c_int, C.c_void_p]
        L.orc_mcc.restype = C.c_int64
        L.orc_boris.argtypes = [_dp, _dp, C.c_double, C.c_double, _dp]
        L.orc_boris.restype = None

    @contextlib.contextmanager
    def _scan(self, mesh):
        """Select the scan accelerator of `mesh` for the calls inside (fast_locate only)."""
        if not self.fast_locate:
            yield
            return
        key = id(mesh)
        if key not in self._grids:
            self._grids[key] = (mesh, self.L.orc_grid_create(mesh.xyz, mesh.tet, mesh.T))
        self.L.orc_grid_use(self._grids[key][1])
        try:
            yield
        finally:
            self.L.orc_grid_use(None)

    def close(self):
        for _, g in self._grids.values():
            self.L.orc_grid_destroy(g)
        self._grids.clear()

    # -- RNG
    def philox(self, ctr, key):
        o = np.zeros(4, dtype=np.uint32)
        self.L.orc_philox4x32_10(np.asarray(ctr, np.uint32), np.asarray(key, np.uint32), o)
        return o

    # -- geometry
    def barycentric(self, mesh, t, p):
        lam = np.zeros(4)
        ok = self.L.orc_barycentric(mesh.xyz, mesh.tet, int(t), np.asarray(p, np.float64), lam)
        return bool(ok), lam

    def locate(self, mesh, p, hint=-1, neighbors=True):
        nb = _nullable(mesh.nbr, np.int32) if neighbors else None
        with self._scan(mesh):
            return int(self.L.orc_locate_point(mesh.xyz, mesh.tet, nb, mesh.T, np.asarray(p, np.float64), int(hint)))

    # -- push
    def push(self, mesh, E, parts, species, dt, nseg=10, kernel=1, deposit=True, neighbors=True,
             floor_ratio=0.001, status=None):
        P = parts["x"].shape[0]
        x = parts["x"].copy()
        v = parts["v"].copy()
        tet = parts["tet"].astype(np.int32).copy()
        st = np.zeros(P, np.uint8) if status is None else status.astype(np.uint8).copy()
        lost = np.zeros(P, np.uint8)
        sq = np.array([s.q for s in species])
        sm = np.array([s.m for s in species])
        sw = np.array([s.w for s in species])
        rho = np.zeros(mesh.N)
        pp = PushParams(dt, floor_ratio, nseg, kernel, 1 if deposit else 0, 0)
        stats = PushStats()
        nb = _nullable(mesh.nbr, np.int32) if neighbors else None
        with self._scan(mesh):
            self.L.orc_push(mesh.N, mesh.xyz, mesh.T, mesh.tet, nb, np.ascontiguousarray(E, np.float64).reshape(-1),
                            P, x.reshape(-1), v.reshape(-1), parts["species"].astype(np.int32), tet, st, lost, sq, sm,
                            sw, C.byref(pp), rho, C.byref(stats))
        return dict(x=x, v=v, tet=tet, lost=lost, status=st, rho=rho, substeps=stats.substeps,
                    nlost=stats.lost)

    def boundary(self, mesh, out, parts, species, face_bc, period=(0.0, 0.0, 0.0), neighbors=True,
                 body_tally=False):
        P = out["x"].shape[0]
        b = BcParams()
        lo, hi = mesh.xyz.min(axis=0), mesh.xyz.max(axis=0)
        for a in range(3):
            b.bmin[a] = lo[a]
            b.bmax[a] = hi[a]
            b.period[a] = period[a]
        for f in range(6):
            b.face_bc[f] = face_bc[f]
        b.body_tally = 1 if body_tally else 0
        ledger = np.zeros(7 * 8)
        sc = np.zeros(1)
        sq = np.array([s.q for s in species])
        sm = np.array([s.m for s in species])
        sw = np.array([s.w for s in species])
        nb = _nullable(mesh.nbr, np.int32) if neighbors else None
        with self._scan(mesh):
            self.L.orc_boundary(mesh.T, mesh.xyz, mesh.tet, nb, P, out["x"].reshape(-1), out["v"].reshape(-1),
                                parts["species"].astype(np.int32), out["tet"], out["status"], out["lost"], sq, sm, sw,
                                C.byref(b), ledger, sc)
        out["ledger"] = ledger.reshape(7, 8)
        out["surface_charge"] = float(sc[0])
        return out

    # -- field solve
    def assemble(self, mesh, eps_tet=None):
        N = mesh.N
        rowptr = np.zeros(N + 1, np.int64)
        nnz = C.c_int64()
        self.L.orc_assemble(N, mesh.xyz, mesh.T, mesh.tet, _nullable(eps_tet, np.float64), rowptr, None, None,
                            None, None, C.byref(nnz))
        col = np.zeros(nnz.value, np.int32)
        offw = np.zeros(nnz.value)
        diag = np.zeros(N)
        cv = np.zeros(N)
        self.L.orc_assemble(N, mesh.xyz, mesh.T, mesh.tet, _nullable(eps_tet, np.float64), rowptr,
                            col.ctypes.data_as(C.c_void_p), offw.ctypes.data_as(C.c_void_p),
                            diag.ctypes.data_as(C.c_void_p), cv.ctypes.data_as(C.c_void_p), C.byref(nnz))
        return dict(rowptr=rowptr, col=col, offw=offw, diag=diag, cv=cv)

    def poisson(self, mesh, A, rho, phi_bc, rtol=1e-15, max_iter=20000, charge_sign=-1.0, phi0=None):
        phi = (phi_bc if phi0 is None else phi0).astype(np.float64).copy()
        phi[mesh.dirichlet == 1] = phi_bc[mesh.dirichlet == 1]
        rel = C.c_double()
        it = self.L.orc_poisson_cg(mesh.N, A["rowptr"], A["col"], A["offw"], A["diag"], A["cv"], mesh.dirichlet,
                                   np.ascontiguousarray(rho, np.float64), charge_sign, phi, rtol, max_iter,
                                   C.byref(rel))
        return phi, it, rel.value

    def lsq(self, mesh, A, phi, reg=0.0):
        E = np.zeros(mesh.N * 3)
        self.L.orc_lsq_efield(mesh.N, mesh.xyz, A["rowptr"], A["col"], np.ascontiguousarray(phi, np.float64), reg,
                              E)
        return E.reshape(-1, 3)

    def mcc(self, v, species_idx, status, ids, species, procs, dt, seed, step, mode=0, vmax=None):
        """vmax (mode 2): per species, the largest speed of the previous push (None: none yet)."""
        v = v.copy()
        sm = np.array([s.m for s in species])
        arr = (Elastic * len(procs))(*procs)
        vm = None if vmax is None else np.ascontiguousarray(vmax, np.float64)
        hits = self.L.orc_mcc(v.shape[0], v.reshape(-1), species_idx.astype(np.int32), status.astype(np.uint8),
                              ids.astype(np.int64), sm, arr, dt, seed, step, mode,
                              None if vm is None else vm.ctypes.data_as(C.c_void_p))
        return v, int(hits)


def push_speed_bound(v, species_idx, status, nspecies):
    """The device's null-collision speed bound of each species after a push: the largest
    squared speed of the active particles rounded to FP32, its FP32 square root."""
    out = np.zeros(nspecies)
    v2 = np.sum(np.asarray(v, np.float64) ** 2, axis=1).astype(np.float32)
    for s in range(nspecies):
        m = (species_idx == s) & (status == ACTIVE)
        if m.any():
            out[s] = float(np.sqrt(np.float32(v2[m].max()), dtype=np.float32))
    return out


# ---------------------------------------------------------------------------------------
# Reference (compiled from the reference sources)
# ---------------------------------------------------------------------------------------
def reference_available(omp: bool = False) -> bool:
    return os.path.exists(REF_OMP_SO if omp else REF_SO)


class Reference:
    def __init__(self, omp: bool = False):
        L = C.CDLL(REF_OMP_SO if omp else REF_SO)
        self.L = L
        L.ref_mesh_create.argtypes = [C.c_int64, _dp, C.c_int64, _i32p, C.c_void_p, _u8p]
        L.ref_mesh_create.restype = C.c_void_p
        L.ref_mesh_destroy.argtypes = [C.c_void_p]
        L.ref_push.argtypes = [C.c_void_p, _dp, C.c_int64, _dp, _dp, _i32p, _dp, _i32p, _u8p, C.c_double, C.c_int,
                               C.c_int, _dp, C.POINTER(C.c_int64)]
        L.ref_poisson.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.ref_push_parallel.argtypes = [C.c_void_p, _dp, C.c_int64, _dp, _dp, _i32p, _dp, _i32p, _u8p, C.c_double,
                                        C.c_int, C.c_int, _dp, C.POINTER(C.c_int)]
        L.ref_push_parallel.restype = C.c_double
        L.ref_lsq_field.argtypes = [C.c_void_p, _dp, _dp]
        L.ref_cycle_run.argtypes = [C.c_void_p, C.c_int64, _dp, _dp, _i32p, _dp, _i32p, C.c_int, C.c_double, _i32p,
                                    _dp, C.POINTER(C.c_int64), _i64p, _i32p, _dp, _dp, _dp, _dp, _dp, _dp]
        L.ref_cycle_mcc_run.argtypes = [C.c_void_p, C.c_int64, _dp, _dp, _i32p, _dp, _i32p, C.c_int, C.c_double,
                                        _i32p, _dp, C.c_double, C.c_double, C.c_uint, C.POINTER(C.c_int64), _i64p,
                                        _i32p, _dp, _dp, _dp, _dp, _dp, C.POINTER(C.c_int64)]
        L.ref_mcc_count.argtypes = [C.c_int64, _dp, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                    C.c_uint, C.c_int, C.POINTER(C.c_int64)]
        L.ref_mcc_count.restype = C.c_int64
        L.ref_circuit_advance.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_double, _dp]
        L.ref_circuit_advance.restype = C.c_int
        L.ref_whipple_yield.argtypes = [C.c_double, C.c_double, C.c_int, _dp, _dp]
        L.ref_whipple_yield.restype = None
        L.ref_legacy_yield.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_int, _dp, _dp]
        L.ref_legacy_yield.restype = None
        L.ref_parse_cross_section_set.argtypes = [C.c_char_p]
        L.ref_parse_cross_section_set.restype = C.c_int
        L.ref_estimate_densities.argtypes = [C.c_int64, _i32p, _dp, _dp, _u8p, C.c_double, _dp, _dp]
        L.ref_estimate_densities.restype = None
        L.ref_sampler_mesh.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, C.c_int64, _dp, C.c_int64, _i32p,
                                       _i64p]
        L.ref_sampler_mesh.restype = C.c_int
        L.ref_sampler_sample.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_uint] + \
            [C.c_double] * 8 + [C.c_int, _dp]
        L.ref_sampler_sample.restype = C.c_int
        L.ref_csv_export.argtypes = [C.c_char_p, C.c_char_p, C.c_int64, _dp, C.c_int, C.POINTER(C.c_char_p),
                                     C.POINTER(C.c_void_p)]
        L.ref_csv_export.restype = C.c_int
        self._meshes = {}

    def mesh(self, mesh: BoxMesh, neighbors=True):
        key = (id(mesh), neighbors)
        if key not in self._meshes:
            nb = _nullable(mesh.nbr, np.int32) if neighbors else None
            self._meshes[key] = (mesh, self.L.ref_mesh_create(mesh.N, mesh.xyz, mesh.T, mesh.tet, nb, mesh.dirichlet))
        return self._meshes[key][1]

    def close(self):
        for _, h in self._meshes.values():
            self.L.ref_mesh_destroy(h)
        self._meshes.clear()

    def push(self, mesh, E, parts, species, dt, nseg=10, kernel=1, neighbors=True):
        h = self.mesh(mesh, neighbors)
        P = parts["x"].shape[0]
        x = parts["x"].copy()
        v = parts["v"].copy()
        kind = np.array([species[s].kind for s in parts["species"]], np.int32)
        w = np.array([species[s].w for s in parts["species"]], np.float64)
        tet = parts["tet"].astype(np.int32).copy()
        lost = np.zeros(P, np.uint8)
        rho = np.zeros(mesh.N)
        sub = C.c_int64()
        self.L.ref_push(h, np.ascontiguousarray(E, np.float64).reshape(-1), P, x.reshape(-1), v.reshape(-1), kind, w,
                        tet, lost, dt, nseg, kernel, rho, C.byref(sub))
        return dict(x=x, v=v, tet=tet, lost=lost, rho=rho, substeps=sub.value)

    def push_parallel(self, mesh, E, parts, species, dt, nseg=10, kernel=1):
        """Reference push over all host threads; returns (result dict, seconds, threads)."""
        h = self.mesh(mesh, True)
        P = parts["x"].shape[0]
        x = parts["x"].copy()
        v = parts["v"].copy()
        kind = np.array([species[s].kind for s in parts["species"]], np.int32)
        w = np.array([species[s].w for s in parts["species"]], np.float64)
        tet = parts["tet"].astype(np.int32).copy()
        lost = np.zeros(P, np.uint8)
        rho = np.zeros(mesh.N)
        nt = C.c_int()
        secs = self.L.ref_push_parallel(h, np.ascontiguousarray(E, np.float64).reshape(-1), P, x.reshape(-1),
                                        v.reshape(-1), kind, w, tet, lost, dt, nseg, kernel, rho, C.byref(nt))
        return dict(x=x, v=v, tet=tet, lost=lost, rho=rho), float(secs), nt.value

    def poisson(self, mesh, rho, phi_bc):
        h = self.mesh(mesh)
        phi = phi_bc.astype(np.float64).copy()
        E = np.zeros(mesh.N * 3)
        rc = self.L.ref_poisson(h, np.ascontiguousarray(rho, np.float64), phi, E)
        assert rc == 0
        return phi, E.reshape(-1, 3)

    def lsq(self, mesh, phi):
        h = self.mesh(mesh)
        E = np.zeros(mesh.N * 3)
        self.L.ref_lsq_field(h, np.ascontiguousarray(phi, np.float64), E)
        return E.reshape(-1, 3)

    def cycle(self, mesh, parts, species, nsteps, dt, face_bc, phi0, neighbors=True):
        h = self.mesh(mesh, neighbors)
        P = parts["x"].shape[0]
        x = parts["x"].copy()
        v = parts["v"].copy()
        kind = np.array([species[s].kind for s in parts["species"]], np.int32)
        w = np.array([species[s].w for s in parts["species"]], np.float64)
        Pout = C.c_int64()
        ids = np.zeros(P, np.int64)
        status = np.zeros(P, np.int32)
        rho = np.zeros(mesh.N)
        phi = np.zeros(mesh.N)
        E = np.zeros(mesh.N * 3)
        ledger = np.zeros(6 * 8)
        stats = np.zeros(5)
        secs = np.zeros(1)
        rc = self.L.ref_cycle_run(h, P, x.reshape(-1), v.reshape(-1), kind, w, parts["tet"].astype(np.int32),
                                  nsteps, dt, np.asarray(face_bc, np.int32), np.ascontiguousarray(phi0, np.float64),
                                  C.byref(Pout), ids, status, rho, phi, E, ledger, stats, secs)
        assert rc == 0, rc
        return dict(x=x, v=v, id=ids[:Pout.value] - 1, status=status, rho=rho, phi=phi, E=E.reshape(-1, 3),
                    ledger=ledger.reshape(6, 8), stats=stats, seconds=float(secs[0]))

    def cycle_mcc(self, mesh, parts, species, nsteps, dt, face_bc, phi0, n_target, sigma, seed, neighbors=True):
        """PICCycle steps, each followed by Collision::executeBackgroundMccStep with a constant
        elastic cross-section for both species (ref_harness.cpp: ref_cycle_mcc_run).  The
        container drops inactive particles after every MCC step: only active particles return,
        with their 0-based ids."""
        h = self.mesh(mesh, neighbors)
        P = parts["x"].shape[0]
        x = parts["x"].copy()
        v = parts["v"].copy()
        kind = np.array([species[s].kind for s in parts["species"]], np.int32)
        w = np.array([species[s].w for s in parts["species"]], np.float64)
        Pout, hits = C.c_int64(), C.c_int64()
        ids = np.zeros(P, np.int64)
        status = np.zeros(P, np.int32)
        rho, phi, E = np.zeros(mesh.N), np.zeros(mesh.N), np.zeros(mesh.N * 3)
        ledger, stats = np.zeros(6 * 8), np.zeros(5)
        rc = self.L.ref_cycle_mcc_run(h, P, x.reshape(-1), v.reshape(-1), kind, w, parts["tet"].astype(np.int32),
                                      nsteps, dt, np.asarray(face_bc, np.int32), np.ascontiguousarray(phi0, np.float64),
                                      n_target, sigma, seed, C.byref(Pout), ids, status, rho, phi, E, ledger, stats,
                                      C.byref(hits))
        assert rc == 0, rc
        n = Pout.value
        return dict(x=x[:n], v=v[:n], id=ids[:n] - 1, status=status[:n], rho=rho, phi=phi, E=E.reshape(-1, 3),
                    ledger=ledger.reshape(6, 8), stats=stats, hits=hits.value)

    def circuit_advance(self, C_f, G_s, V0, I_a, didv, dt):
        """SurfaceCircuitCoupling::advanceImplicit over independent nodes: the new potentials."""
        a = [np.ascontiguousarray(v, np.float64) for v in (C_f, G_s, V0, I_a, didv)]
        out = np.zeros(len(a[0]))
        assert self.L.ref_circuit_advance(len(out), *a, float(dt), out) == 0
        return out

    def whipple_yield(self, peak_yield, peak_energy_ev, e_ev):
        """evaluateLegacySecondaryElectronYield(Whipple) of a material with these peaks."""
        e = np.ascontiguousarray(e_ev, np.float64)
        out = np.zeros(len(e))
        self.L.ref_whipple_yield(float(peak_yield), float(peak_energy_ev), len(e), e, out)
        return out

    def sampler_mesh(self, area_m2, aspect, gap_m, z_layers):
        """The surface current sampler's plate mesh (GeometryMeshGenerator, as createSamplingMesh
        builds it for a sampler with no linked boundary faces): node coordinates and tets."""
        cap = 100000
        xyz = np.zeros((cap, 3))
        tet = np.zeros((cap, 4), np.int32)
        cnt = np.zeros(2, np.int64)
        assert self.L.ref_sampler_mesh(float(area_m2), float(aspect), float(gap_m), int(z_layers), cap, xyz, cap, tet,
                                       cnt) == 0
        return xyz[:cnt[0]].copy(), tet[:cnt[1]].copy()

    def sampler_sample(self, area_m2, gap_m, z_layers, ppe, window_steps, seed, ne, ni, te_ev, ti_ev, ion_amu,
                       surface_v, reference_v, probe_dv, enable_mcc=False):
        """PicMccSurfaceCurrentSampler::sampleWithDerivative: electron, ion, emitted and net
        collection current densities [A/m^2], d(net)/dV, valid, deposition segments, seed used."""
        out = np.zeros(8)
        self.L.ref_sampler_sample(float(area_m2), float(gap_m), int(z_layers), int(ppe), int(window_steps), int(seed),
                                  float(ne), float(ni), float(te_ev), float(ti_ev), float(ion_amu), float(surface_v),
                                  float(reference_v), float(probe_dv), int(bool(enable_mcc)), out)
        keys = ("electron", "ion", "emitted", "net", "derivative", "valid", "segments", "seed")
        return dict(zip(keys, out))

    def csv_export(self, path, axis_name, axis, series):
        """CSVExporter::exportDataSet of {name: values} over the axis; True on success."""
        names = list(series)
        vals = [np.ascontiguousarray(series[k], np.float64) for k in names]
        cn = (C.c_char_p * max(1, len(names)))(*[k.encode() for k in names])
        cv = (C.c_void_p * max(1, len(names)))(*[v.ctypes.data for v in vals])
        a = np.ascontiguousarray(axis, np.float64)
        return self.L.ref_csv_export(str(path).encode(), axis_name.encode(), len(a), a, len(names), cn, cv) == 0

    def legacy_yield(self, model, peak_yield, peak_energy_ev, e_ev, sims_n=1.6, katz=None):
        """evaluateLegacySecondaryElectronYield, model "whipple", "sims" or "katz"."""
        e = np.ascontiguousarray(e_ev, np.float64)
        out = np.zeros(len(e))
        k = None if katz is None else np.ascontiguousarray(katz, np.float64)
        self.L.ref_legacy_yield({"whipple": 0, "sims": 1, "katz": 2}[model], float(peak_yield), float(peak_energy_ev),
                                float(sims_n), None if k is None else k.ctypes.data, len(e), e, out)
        return out

    def parse_cross_section_set(self, text):
        """Collision::parseCollisionCrossSectionSetId: -1 unknown, else the set's index."""
        return int(self.L.ref_parse_cross_section_set(text.encode()))

    def estimate_densities(self, types, charges, weights, active, volume, floors):
        """Collision::estimateCollisionBackgroundDensities: (neutral, ion, electron) densities."""
        out = np.zeros(3)
        self.L.ref_estimate_densities(len(types), np.ascontiguousarray(types, np.int32),
                                      np.ascontiguousarray(charges, np.float64),
                                      np.ascontiguousarray(weights, np.float64),
                                      np.ascontiguousarray(active, np.uint8), float(volume),
                                      np.ascontiguousarray(floors, np.float64), out)
        return out

    def mcc_count(self, v, kind, w, sigma, n_target, dt, seed, repeats):
        """(first-draw hits as the handler counts them, particles actually scattered)"""
        sc = C.c_int64()
        hits = int(self.L.ref_mcc_count(v.shape[0], np.ascontiguousarray(v, np.float64).reshape(-1), kind, w, sigma,
                                        n_target, dt, seed, repeats, C.byref(sc)))
        return hits, sc.value


# ----------------------------------------------------------------------------------------
# Surface circuit of the body faces (restated for the parity tests; no reference test covers
# an interior body, so these follow the device rule and the reference's node update)
# ----------------------------------------------------------------------------------------
EPS0 = 8.8541878128e-12


def body_face_of(x, blo, bhi):
    """Face XMin..ZMax of the body box nearest to each position (ties: the lowest face)."""
    d = np.stack([np.abs(x[:, 0] - blo[0]), np.abs(bhi[0] - x[:, 0]), np.abs(x[:, 1] - blo[1]),
                  np.abs(bhi[1] - x[:, 1]), np.abs(x[:, 2] - blo[2]), np.abs(bhi[2] - x[:, 2])], axis=1)
    return np.argmin(d, axis=1)


def sims_xm(n):
    """The root xm of the Sims yield for exponent n, by legacySimsYield's own grid search
    (Tools/Material/src/SurfaceMaterialModel.cpp:252-263)."""
    for i in range(1, 10001):
        x = 0.5 + i * (2.5 - 0.5) / 10000.0
        if abs(x - (1.0 - 1.0 / n) * (math.exp(x) - 1.0)) <= 1.0e-3:
            return x
    return 2.5


def see_yield(model, dmax, emax, e_ev, sims_n=1.6, katz=(0.85, 0.35, 0.12, 1.05)):
    """Secondary-electron yield: 1 Sternglass 7.4 dmax (E/Emax) exp(-2 sqrt(E/Emax)); the
    reference's legacy yields (Tools/Material/src/SurfaceMaterialModel.cpp): 2 legacyWhippleYield
    (:231-244), 3 legacySimsYield (:246-273), 4 legacyKatzYield (:275-302)."""
    e = np.asarray(e_ev, float)
    out = np.zeros_like(e)
    ok = (e > 0) & (dmax > 0)
    if model == 3:
        n = max(1.05, sims_n)
        xm = sims_xm(n)
        ep = max(1.0, emax)
        ok &= e > 10.0
        x = xm * (e[ok] / ep) ** n
        good = (x > 1e-12) & (abs(1.0 - math.exp(-xm)) >= 1e-12)
        xs = np.where(good, x, 1.0)
        out[ok] = np.where(good, dmax / (1.0 - math.exp(-xm)) * (ep / e[ok]) ** (n - 1.0) * 2.0
                           * (xs + np.exp(-xs) - 1.0) / xs, 0.0)
        return out
    if model == 4:
        ok = (e > 1e-9) & (dmax > 0)
        ep = max(1.0, emax)
        r1, n1, r2, n2 = katz
        ek, pk = e[ok] * 1e-3, ep * 1e-3
        rng = r1 * ek ** n1 + r2 * ek ** n2
        prng = r1 * pk ** n1 + r2 * pk ** n2
        good = (rng > 1e-12) & (prng > 1e-12)
        att = np.exp(-(rng / prng - 1.0) ** 2)
        roll = 1.0 / (1.0 + (e[ok] / max(1.0, 3.0 * ep)) ** 0.7)
        out[ok] = np.where(good, dmax * att * (0.55 + 0.45 * roll), 0.0)
        return out
    if model == 1:
        r = e[ok] / emax
        out[ok] = 7.4 * dmax * r * np.exp(-2.0 * np.sqrt(r))
    elif model == 2:
        ep = max(1.0, emax)
        q = 2.28 * (e[ok] / ep) ** 1.35
        v = np.where(q > 1e-12, 2.228 * (q - 1.0 + np.exp(-q)) / np.where(q > 1e-12, q, 1.0) * dmax
                     * (ep / e[ok]) ** 0.35, 0.0)
        out[ok] = v
    return out


class SurfaceCircuit:
    """Faces of the body box as circuit nodes, C = eps0 eps_r A / d
    (DensePlasmaSurfaceCharging.cpp:6544-6552), advanced per step by the implicit node update
    of SurfaceCircuitCoupling::advanceImplicit (SurfaceCircuitCoupling.cpp:953-966):
    (C/dt + G - dI/dV) V' = C/dt V + I - dI/dV V with I = dq/dt."""

    def __init__(self, mesh, blo, bhi, eps_r=3.0, thickness=1e-3, v0=0.0, shunt=0.0, didv=0.0):
        self.blo, self.bhi = np.asarray(blo, float), np.asarray(bhi, float)
        ext = self.bhi - self.blo
        area = np.array([ext[(f // 2 + 1) % 3] * ext[(f // 2 + 2) % 3] for f in range(6)])
        b = lambda v: np.broadcast_to(np.asarray(v, float), (6,)).copy()
        self.C = EPS0 * b(eps_r) * area / b(thickness)
        self.G, self.didv, self.V = b(shunt), b(didv), b(v0)
        self.Q = np.zeros(6)
        tol = 1e-9 * ext.max()
        p = mesh.xyz
        inside = np.all((p >= self.blo - tol) & (p <= self.bhi + tol), axis=1) & (mesh.dirichlet == 1)
        masks = np.zeros(mesh.N, np.int64)
        for f in range(6):
            a = f // 2
            plane = self.bhi[a] if f & 1 else self.blo[a]
            masks |= (inside & (np.abs(p[:, a] - plane) <= tol)).astype(np.int64) << f
        self.nodes = np.nonzero(masks)[0]
        self.masks = masks[self.nodes]

    see = (0, 0.0, 300.0)  # (model, delta_max, e_max_ev)

    def collect(self, x_lost, q_lost, e_ev=None, electron=None):
        """Charge of this step's particles lost into the body per face, plus the charge their
        secondaries leave behind; also returns the emitted electrons' charge (negative)."""
        dq = np.zeros(6)
        emitted = 0.0
        if len(q_lost):
            face = body_face_of(x_lost, self.blo, self.bhi)
            np.add.at(dq, face, q_lost)
            if self.see[0] and e_ev is not None:
                em = see_yield(self.see[0], self.see[1], self.see[2], e_ev) * np.abs(q_lost) * electron
                np.add.at(dq, face, em)
                emitted = -float(em.sum())
        return dq, emitted

    def advance(self, dq, dt):
        self.Q += dq
        I = dq / dt
        cdt = self.C / dt
        den = cdt + self.G - self.didv
        ok = den > 0
        self.V[ok] = ((cdt * self.V + I - self.didv * self.V) / np.where(ok, den, 1.0))[ok]

    def apply(self, phi):
        for i, m in zip(self.nodes, self.masks):
            faces = [f for f in range(6) if (m >> f) & 1]
            s = 0.0
            for f in faces:
                s += self.V[f]
            phi[i] = s / len(faces)
        return phi


def seed_tets(mesh, species_index, n_species, n_per_tet, sigma, seed, tets=None, drift=(0.0, 0.0, 0.0)):
    """Restated samplePointInTetra injection (PicMccSurfaceCurrentSampler.cpp:270-287) with the
    Philox draws of scdat_seed_tet_particles: positions, velocities and tets of every particle."""
    tl = np.arange(mesh.T) if tets is None else np.asarray(tets)
    c = np.repeat(np.arange(len(tl)), n_per_tet)
    j = np.tile(np.arange(n_per_tet), len(tl))
    ids = ((c * n_species + species_index) * n_per_tet + j).astype(np.uint64)
    u01, u23 = uniforms2(seed, ids, 0, 0), uniforms2(seed, ids, 0, 1)
    g01, g23 = uniforms2(seed, ids, 0, 4), uniforms2(seed, ids, 0, 5)
    u = np.concatenate([u01, u23], axis=1)
    e = -np.log(np.maximum(1e-12, u))
    es = ((e[:, 0] + e[:, 1]) + e[:, 2]) + e[:, 3]
    t = tl[c]
    x = np.zeros((len(ids), 3))
    for q in range(4):
        x += (e[:, q] / es)[:, None] * mesh.xyz[mesh.tet[t, q]]
    r1, r2 = np.sqrt(-2.0 * np.log(g01[:, 0])), np.sqrt(-2.0 * np.log(g23[:, 0]))
    tp = 6.283185307179586476925286766559
    v = np.stack([drift[0] + sigma * r1 * np.cos(tp * g01[:, 1]), drift[1] + sigma * r1 * np.sin(tp * g01[:, 1]),
                  drift[2] + sigma * r2 * np.cos(tp * g23[:, 1])], axis=1)
    return x, v, t.astype(np.int32)
