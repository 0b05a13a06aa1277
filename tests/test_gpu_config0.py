"""The first benchmark configuration at its full size, on the device, through the C ABI.

32^3 hex cells of 0.05 m x 6 tets (193,536 tets after the 8^3-cell body, 35,937 nodes), the
body at -10 V and the outer faces at 0 V, electrons and H+ at 1e10 m^-3 and 1 eV, 20
particles per cell per species (1,290,240 particles), dt = 2e-8 s, elastic MCC against
1e14 m^-3 with a constant 1e-19 m^2, Jacobi-PCG.

* the FP64 push of a 4,096-particle subsample against the reference's own CrossTetrahedron
  (tests/golden/config0_ref.npz, made by the reference through oracle/ref_harness.cpp):
  positions and velocities to 1e-12, tets, lost flags and sub-step count exact, charge 1e-12;
* the FP64 push of the whole population against the C oracle: the same bar, per species;
* the field solve from the deposited charge at the configuration's tolerance (1e-8) and at
  1e-14 against the oracle's Jacobi-PCG;
* three full PIC-MCC steps against the oracle's run in the reference's order on the same
  Philox streams: collisions, survivors and ledger counts exact, states and fields to 1e-12;
* the precision form at 48^3 against the FP64 form from the same seeded state.
"""
import os

import numpy as np
import pytest

import oracle as O
from conftest import rel_err
from golden.make_golden import CONFIG0_STRIDE, config0_laplace, make_config0_inputs, subsample
from pic_helpers import gpu_domain, gpu_load_particles, gpu_state, oracle_mcc_run

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-12
FACE_BC = (1,) * 6  # absorbing outer faces


def state_in_order(dom, nspecies, ids):
    """Device particles in the order of `ids` (the particle ids they were uploaded with)."""
    order = np.argsort(ids)
    n = len(ids)
    out = dict(x=np.full((n, 3), np.nan), v=np.full((n, 3), np.nan), tet=np.full(n, -9, np.int32),
               status=np.full(n, 255, np.uint8))
    for s in range(nspecies):
        p = dom.get_particles(s)
        k = order[np.searchsorted(ids[order], p["id"].astype(np.int64))]
        for key in out:
            out[key][k] = p[key]
    return out


@pytest.fixture(scope="module")
def cfg0(lib):
    o = O.Oracle(fast_locate=True)
    mesh, sp, parts, dt = make_config0_inputs()
    A, phi = config0_laplace(o, mesh)
    E = o.lsq(mesh, A, phi, reg=1e-18)
    yield dict(o=o, mesh=mesh, sp=sp, parts=parts, dt=dt, A=A, phi=phi, E=E)
    o.close()


def test_config0_push_matches_reference(cfg0):
    g = np.load(os.path.join(GOLDEN, "config0_ref.npz"))
    mesh, sp, dt = cfg0["mesh"], cfg0["sp"], cfg0["dt"]
    phi = cfg0["phi"]
    # the Laplace potential is recomputed here; it must be the one the fixture was made with
    assert np.sum(phi) == g["phi_sum"] and np.sum(np.abs(phi)) == g["phi_abs_sum"]
    sub = subsample(cfg0["parts"], CONFIG0_STRIDE)
    dom = gpu_domain(mesh, dt)
    gpu_load_particles(dom, sp, sub)
    dom.set_potential(phi)  # PICCycle::setPotential: the device's LSQ field of phi
    _, _, Ed = dom.fields()
    assert abs(np.sum(np.abs(Ed)) - g["E_abs_sum"]) <= TOL * g["E_abs_sum"]
    dom.push()
    n = sub["x"].shape[0]
    st = state_in_order(dom, len(sp), sub["id"])
    lost = g["push_lost"] == 1
    assert lost.sum() < n // 10
    assert np.array_equal(st["status"] != O.ACTIVE, lost)
    assert np.array_equal(st["tet"][~lost], g["push_tet"][~lost])
    assert np.abs(st["x"] - g["push_x"]).max() <= TOL * np.abs(g["push_x"]).max()
    assert rel_err(st["v"], g["push_v"]) < TOL
    assert dom.stats()["substeps"] == int(g["push_substeps"])
    rho, _, _ = dom.fields()
    ref_rho = np.zeros(mesh.N)
    ref_rho[g["rho_nodes"]] = g["rho_vals"]
    assert rel_err(rho, ref_rho) < TOL
    dom.close()


def test_config0_population_push_matches_oracle(cfg0):
    o, mesh, sp, parts, dt = cfg0["o"], cfg0["mesh"], cfg0["sp"], cfg0["parts"], cfg0["dt"]
    P = parts["x"].shape[0]
    assert P == 1290240 and mesh.T == 193536 and mesh.N == 35937
    dom = gpu_domain(mesh, dt)
    gpu_load_particles(dom, sp, parts)
    dom.set_potential(cfg0["phi"])
    dom.push()
    st = gpu_state(dom, len(sp), P)
    ref = o.push(mesh, cfg0["E"], parts, sp, dt)
    lost = ref["lost"] == 1
    assert 0 < lost.sum() < P // 20
    assert np.array_equal(st["status"] != O.ACTIVE, lost)
    assert np.array_equal(st["tet"][~lost], ref["tet"][~lost])
    assert np.abs(st["x"] - ref["x"]).max() <= TOL * np.abs(ref["x"]).max()
    assert rel_err(st["v"], ref["v"]) < TOL
    assert dom.stats()["substeps"] == ref["substeps"]
    for s in range(len(sp)):
        sub = {k: v[parts["species"] == s] for k, v in parts.items()}
        ref_s = o.push(mesh, cfg0["E"], sub, sp, dt)["rho"]
        assert rel_err(dom.species_charge(s), ref_s) < TOL
    rho, _, _ = dom.fields()
    assert rel_err(rho, ref["rho"]) < TOL
    cfg0["rho_push"] = ref["rho"]
    dom.close()


@pytest.mark.parametrize("rtol", [1e-8, 1e-14])
def test_config0_field_solve_matches_oracle(cfg0, rtol):
    """Jacobi-PCG from the Laplace potential with the pushed charge.  At 1e-14 the potentials
    agree to 1e-12; at the configuration's 1e-8 both solves stop within one iteration of each
    other and their potentials differ by far less than the tolerance allows (1e-9 of max|phi|)."""
    o, mesh, A = cfg0["o"], cfg0["mesh"], cfg0["A"]
    rho = cfg0.get("rho_push")
    if rho is None:
        rho = o.push(mesh, cfg0["E"], cfg0["parts"], cfg0["sp"], cfg0["dt"])["rho"]
    ref_phi, ref_it, ref_rel = o.poisson(mesh, A, rho, mesh.phi_bc, rtol=rtol, phi0=cfg0["phi"])
    ref_E = o.lsq(mesh, A, ref_phi)
    dom = gpu_domain(mesh, cfg0["dt"], pcg_rtol=rtol, pcg_max_iter=20000)
    dom.set_species(cfg0["sp"])
    dom.set_potential(cfg0["phi"])
    dom.set_charge_density(rho)
    dom.solve_field(allow_not_converged=rtol < 1e-13)
    _, phi, E = dom.fields()
    it = dom.stats()["last_pcg_iterations"]
    dom.close()
    assert ref_it > 10  # warm start from the Laplace potential
    if rtol < 1e-13:
        assert rel_err(phi, ref_phi) < TOL
        assert rel_err(E, ref_E) < TOL
    else:
        assert abs(it - ref_it) <= 1 and ref_rel <= rtol
        assert rel_err(phi, ref_phi) < 1e-9
        assert rel_err(E, ref_E) < 1e-7


def test_config0_pic_mcc_steps_match_oracle(cfg0):
    """Three full steps with the configuration's MCC against the oracle's run in the reference's
    order (cycle, MCC, inactive particles dropped) on the same Philox streams (solves to 1e-14,
    where both sides give the same potential to 1e-12)."""
    o, mesh, sp, parts, dt = cfg0["o"], cfg0["mesh"], cfg0["sp"], cfg0["parts"], cfg0["dt"]
    n_t, sigma, seed, nsteps = 1e14, 1e-19, 2024, 3
    ref = oracle_mcc_run(o, mesh, sp, parts, nsteps, dt, FACE_BC, n_t, sigma, seed, rtol=1e-14)
    dom = gpu_domain(mesh, dt, face_bc=FACE_BC, pcg_rtol=1e-14, pcg_max_iter=20000, body_tally=False, seed=seed)
    gpu_load_particles(dom, sp, parts)
    for s in range(len(sp)):
        dom.set_elastic(s, n_t, sigma, mode=0)
    dom.set_potential(mesh.phi_bc)
    dom.step(nsteps)
    st = gpu_state(dom, len(sp), parts["x"].shape[0])
    stats = dom.stats()
    rho, phi, E = dom.fields()
    led = dom.ledger()
    dom.close()
    # at the configuration's neutral density the collision probability per particle and step is
    # n sigma |v| dt ~ 1e-7 for electrons, so a few tenths of a collision are expected over the
    # three steps: both sides must agree on the count (MCC at high density has its own tests)
    assert stats["mcc_collisions"] == ref["hits"]
    ids = ref["parts"]["id"]
    act = np.nonzero(st["status"] == O.ACTIVE)[0]
    assert np.array_equal(np.sort(act), np.sort(ids))
    assert np.abs(st["x"][ids] - ref["parts"]["x"]).max() <= TOL * np.abs(ref["parts"]["x"]).max()
    assert rel_err(st["v"][ids], ref["parts"]["v"]) < TOL
    assert rel_err(rho, ref["rho"]) < TOL
    assert rel_err(phi, ref["phi"]) < TOL
    assert rel_err(E, ref["E"]) < TOL
    assert np.array_equal(led[:6, 4:6], ref["ledger"][:6, 4:6]) and led[:6, 4:6].sum() > 0
    np.testing.assert_allclose(led[:6, [0, 1, 3]], ref["ledger"][:6, [0, 1, 3]], rtol=TOL, atol=1e-30)


def test_precision_form_48cube_vs_fp64(lib):
    """The precision form (FP32 tet-relative push, FP32-SpMV PCG under FP64 refinement) at
    48^3 cells x 6 tets, 32 ppc per species (about 7 M particles), against the FP64 form from
    the same seeded state over 4 steps: potential within 1e-5 of max|phi| (the floating-
    potential bar), total charge per species within 1e-9, per-species charge density within
    1e-3 in the L2 norm, and the two forms lose the same particles but for a few."""
    from scdat_b200 import capi

    n, h, ppc = 48, 0.05, 32
    body = ((18, 30), (18, 30), (18, 30))
    m = capi.kuhn_box_mesh((n, n, n), h, body=body, bias=-10.0)
    sp = O.plasma_species(1e10, 1.0, 1.0, h, ppc)
    out = {}
    for prec in (0, 1):
        dom = capi.Domain(m["xyz"], m["tet"], m["dirichlet"], 2e-8, precision=prec, face_bc=FACE_BC, pcg_rtol=1e-10,
                          pcg_max_iter=20000, sort_interval=1)
        dom.set_species(sp)
        for s in range(2):
            dom.seed_box(s, (n, n, n), h, body, ppc, 1.0, 77)
        dom.set_potential(m["phi"])
        dom.step(4)
        rho, phi, _ = dom.fields()
        out[prec] = dict(phi=phi, rs=[dom.species_charge(s) for s in range(2)], st=dom.stats())
        dom.close()
    a, b = out[0], out[1]
    assert a["st"]["active_particles"] > 6_000_000
    e_phi = rel_err(b["phi"], a["phi"])
    print(f"48^3 mixed vs FP64 after 4 steps: phi {e_phi:.3e} of max|phi|")
    assert e_phi < 1e-5
    for s in range(2):
        ra, rb = a["rs"][s], b["rs"][s]
        dq = abs(rb.sum() - ra.sum()) / np.abs(ra).sum()
        l2 = np.linalg.norm(rb - ra) / np.linalg.norm(ra)
        print(f"  species {s}: total charge {dq:.3e}, charge density L2 {l2:.3e}")
        # the segment-cloud deposit drops sample points outside the post-move tet, so the totals
        # of the two forms differ by the few sample points that FP32 rounding moves across a face
        assert dq <= 1e-6
        assert l2 <= 1e-3
    da = abs(a["st"]["active_particles"] - b["st"]["active_particles"])
    print(f"  active particles: FP64 {a['st']['active_particles']}, mixed {b['st']['active_particles']}")
    assert da <= 1e-4 * a["st"]["active_particles"]
