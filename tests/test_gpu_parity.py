"""CUDA library (through its C ABI) against the reference fixtures and the C oracle.

FP64 form: per-particle state and nodal fields within 1e-12 relative of the reference;
tets, status and counters exact.  Mixed form: error against the FP64 form reported and
bounded.  All inputs are the seeded small cases of tests/golden."""
import os

import numpy as np
import pytest

import oracle as O
from conftest import rel_err
from golden.make_golden import CASES, make_inputs
from pic_helpers import gpu_domain, gpu_load_particles, gpu_state, oracle_cycle, oracle_mcc_run

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-12


@pytest.fixture(params=sorted(CASES))
def case(request, lib):
    return request.param, np.load(os.path.join(GOLDEN, f"{request.param}.npz"))


def test_push_matches_reference(case):
    name, g = case
    mesh, sp, parts, dt, nsteps, face_bc = make_inputs(name)
    dom = gpu_domain(mesh, dt)
    gpu_load_particles(dom, sp, parts)
    dom.set_electric_field(g["E_laplace"])
    dom.push()
    st = gpu_state(dom, len(sp), len(parts["tet"]))
    lost = g["push_lost"] == 1
    assert np.array_equal(st["status"] != O.ACTIVE, lost)
    assert np.array_equal(st["tet"][~lost], g["push_tet"][~lost])
    assert np.abs(st["x"] - g["push_x"]).max() <= TOL * np.abs(g["push_x"]).max()
    assert rel_err(st["v"], g["push_v"]) < TOL
    rho, _, _ = dom.fields()
    assert rel_err(rho, g["push_rho"]) < TOL
    assert dom.stats()["substeps"] == int(g["push_substeps"])
    dom.close()


def test_push_species_charge_matches_oracle(case, orc):
    name, g = case
    mesh, sp, parts, dt, nsteps, face_bc = make_inputs(name)
    dom = gpu_domain(mesh, dt)
    gpu_load_particles(dom, sp, parts)
    dom.set_electric_field(g["E_laplace"])
    dom.push()
    for s in range(len(sp)):
        sub = {k: v[parts["species"] == s] for k, v in parts.items()}
        ref_s = orc.push(mesh, g["E_laplace"], sub, sp, dt)["rho"]
        assert rel_err(dom.species_charge(s), ref_s) < TOL
    dom.close()


def test_poisson_matches_reference(case):
    name, g = case
    mesh, sp, parts, dt, nsteps, face_bc = make_inputs(name)
    dom = gpu_domain(mesh, dt, pcg_rtol=1e-15, pcg_max_iter=20000)
    dom.set_species(sp)
    dom.set_potential(mesh.phi_bc)
    dom.solve_field(allow_not_converged=True)
    _, phi, E = dom.fields()
    assert rel_err(phi, g["phi_laplace"]) < TOL
    assert rel_err(E, g["E_laplace"]) < TOL
    dom.close()


def test_full_cycle_matches_reference(case):
    name, g = case
    mesh, sp, parts, dt, nsteps, face_bc = make_inputs(name)
    dom = gpu_domain(mesh, dt, face_bc=face_bc, pcg_rtol=1e-15, pcg_max_iter=20000, body_tally=False)
    gpu_load_particles(dom, sp, parts)
    dom.set_potential(g["phi_laplace"])
    for _ in range(nsteps):
        dom.step(1)
    st = gpu_state(dom, len(sp), len(parts["tet"]))
    ids = g["cyc_id"]
    smap = {10: O.ACTIVE, 20: O.ABSORBED, 21: O.ESCAPED}
    assert np.array_equal(st["status"][ids], np.array([smap[s] for s in g["cyc_status"]]))
    act = g["cyc_status"] == 10
    assert np.abs(st["x"][ids][act] - g["cyc_x"][act]).max() <= TOL * np.abs(g["cyc_x"]).max()
    assert rel_err(st["v"][ids][act], g["cyc_v"][act]) < TOL
    rho, phi, E = dom.fields()
    assert rel_err(rho, g["cyc_rho"]) < TOL
    assert rel_err(phi, g["cyc_phi"]) < TOL
    assert rel_err(E, g["cyc_E"]) < TOL
    led = dom.ledger()
    assert np.array_equal(led[:6, 4:6], g["cyc_ledger"][:, 4:6])
    np.testing.assert_allclose(led[:6, [0, 1, 3]], g["cyc_ledger"][:, [0, 1, 3]], rtol=TOL, atol=1e-30)
    stt = dom.stats()
    np.testing.assert_allclose(stt["surface_deposited_charge"], g["cyc_stats"][4], rtol=TOL, atol=1e-30)
    np.testing.assert_allclose(stt["total_charge"], g["cyc_stats"][1], rtol=1e-9, atol=1e-12 * np.abs(g["cyc_rho"]).sum())
    np.testing.assert_allclose(stt["total_energy"], g["cyc_stats"][2], rtol=1e-12)
    dom.close()


@pytest.mark.parametrize("neighbors", [True, False])
@pytest.mark.parametrize("kernel", [0, 1, 2])
def test_push_variants_match_oracle(lib, orc, neighbors, kernel):
    mesh, sp, parts, dt, _, _ = make_inputs("box6_body")
    g = np.load(os.path.join(GOLDEN, "box6_body.npz"))
    dom = gpu_domain(mesh, 3e-8, neighbors=neighbors, deposit_kernel=kernel)
    gpu_load_particles(dom, sp, parts)
    dom.set_electric_field(g["E_laplace"] * 5.0)
    dom.push()
    o = orc.push(mesh, g["E_laplace"] * 5.0, parts, sp, 3e-8, kernel=kernel, neighbors=neighbors)
    st = gpu_state(dom, len(sp), len(parts["tet"]))
    lost = o["lost"] == 1
    assert np.array_equal(st["status"] != O.ACTIVE, lost)
    assert np.array_equal(st["tet"][~lost], o["tet"][~lost])
    assert rel_err(st["v"], o["v"]) < TOL
    rho, _, _ = dom.fields()
    assert rel_err(rho, o["rho"]) < TOL
    dom.close()


@pytest.mark.parametrize("mode", [0, 1])
def test_mcc_matches_oracle_streams(lib, orc, mode):
    """Same Philox streams on both sides: identical collision sets, velocities to 1e-12."""
    mesh = O.kuhn_box((4, 4, 4), 0.05)
    sp = O.plasma_species(1e10, 3.0, 3.0, 0.05, 8)
    parts = O.seed_particles(mesh, sp, 8, 21)
    dom = gpu_domain(mesh, 2e-8, seed=4242)
    gpu_load_particles(dom, sp, parts)
    n_t, sigma = 4e20, 1e-19
    for s in range(2):
        dom.set_elastic(s, n_t, sigma, mode=mode)
    dom.collide()
    st = gpu_state(dom, len(sp), len(parts["tet"]))
    procs = [O.Elastic(n_t, sigma, 1.0, 0.0, 0.0, 1, 0) for _ in sp]
    v, hits = orc.mcc(parts["v"], parts["species"], np.zeros(len(parts["tet"]), np.uint8), parts["id"], sp, procs,
                      2e-8, 4242, 0, mode=mode)
    assert dom.stats()["mcc_collisions"] == hits and hits > 50
    changed_g = np.any(st["v"] != parts["v"], axis=1)
    changed_o = np.any(v != parts["v"], axis=1)
    assert np.array_equal(changed_g, changed_o)
    assert rel_err(st["v"], v) < TOL
    dom.close()


@pytest.mark.parametrize("mode", [0, 2])
def test_full_mcc_run_matches_oracle(lib, orc, mode):
    """Several full steps with elastic MCC (fused into the push) against the oracle's run in the
    reference's order (cycle, then MCC, then inactive particles dropped) on the same Philox
    streams: the same collisions, statuses and ledger counts, and states, fields and ledger
    charges to 1e-12.  MCC changes velocities only, so running it inside the push, before the
    field solve, gives the reference order's result."""
    mesh = O.kuhn_box((4, 4, 4), 0.05)
    sp = O.plasma_species(1e10, 1.0, 1.0, 0.05, 8)
    parts = O.seed_particles(mesh, sp, 8, 33)
    vth = np.sqrt(O.QE / O.ME)
    parts["v"][parts["species"] == 0, 0] += 2.0 * vth  # drift into the +x face
    dt, n_t, sigma, seed, nsteps, face_bc = 2e-8, 4e20, 1e-19, 777, 4, (1,) * 6
    ref = oracle_mcc_run(orc, mesh, sp, parts, nsteps, dt, face_bc, n_t, sigma, seed, mode=mode)
    dom = gpu_domain(mesh, dt, face_bc=face_bc, pcg_rtol=1e-15, pcg_max_iter=20000, body_tally=False, seed=seed)
    gpu_load_particles(dom, sp, parts)
    for s in range(len(sp)):
        dom.set_elastic(s, n_t, sigma, mode=mode)
    dom.set_potential(mesh.phi_bc)
    dom.step(nsteps)
    st = gpu_state(dom, len(sp), len(parts["tet"]))
    stats = dom.stats()
    rho, phi, E = dom.fields()
    led = dom.ledger()
    dom.close()
    assert stats["mcc_collisions"] == ref["hits"] and ref["hits"] > 200
    ids = ref["parts"]["id"]
    act = np.nonzero(st["status"] == O.ACTIVE)[0]
    assert np.array_equal(np.sort(act), np.sort(ids))  # the same particles survive
    assert np.abs(st["x"][ids] - ref["parts"]["x"]).max() <= TOL * np.abs(ref["parts"]["x"]).max()
    assert rel_err(st["v"][ids], ref["parts"]["v"]) < TOL
    assert rel_err(rho, ref["rho"]) < TOL
    assert rel_err(phi, ref["phi"]) < TOL
    assert rel_err(E, ref["E"]) < TOL
    assert np.array_equal(led[:6, 4:6], ref["ledger"][:6, 4:6]) and led[1, 4] > 0
    np.testing.assert_allclose(led[:6, [0, 1, 3]], ref["ledger"][:6, [0, 1, 3]], rtol=TOL, atol=1e-30)


def test_picycle_boundary_scenarios(lib):
    """Tools/PICcore/test/PICCycleBoundary_test.cpp:121-221 on the device."""
    mesh = O.kuhn_box((1, 1, 6), 1.0, body=None)
    mesh.xyz[:, 2] /= 6.0
    z = mesh.xyz[:, 2]
    mesh.dirichlet[:] = ((z < 1e-12) | (z > z.max() - 1e-12)).astype(np.uint8)
    sp = [O.Species(-O.QE, O.ME, 1.0, 0, 1.0)]
    cent = mesh.xyz[mesh.tet].mean(axis=1)
    for scen in ("periodic", "absorbing", "far_escape"):
        axis = 0 if scen == "periodic" else 2
        t = int(np.argmax(cent[:, axis]))
        vel = {"periodic": [2e9, 0, 0], "absorbing": [0, 0, 2e9], "far_escape": [0, 0, 5e12]}[scen]
        bc = (0,) * 6 if scen == "far_escape" else (2, 2, 2, 2, 1, 1)
        dom = gpu_domain(mesh, 1e-9, face_bc=bc)
        dom.set_species(sp)
        dom.set_particles(0, cent[t][None, :], np.array([vel], float), np.array([t], np.int32))
        dom.set_potential(np.zeros(mesh.N))
        dom.step(1)
        p = dom.get_particles(0)
        st = dom.stats()
        if scen == "periodic":
            assert p["status"][0] == O.ACTIVE and -1e-9 <= p["x"][0, 0] <= 1.0 + 1e-9
        elif scen == "absorbing":
            led = dom.ledger()
            assert p["status"][0] == O.ABSORBED and st["surface_deposited_charge"] < 0
            assert led[5, 0] < 0 and led[5, 4] == 1
        else:
            assert p["status"][0] != O.ACTIVE and abs(st["surface_deposited_charge"]) < 1e-20
        dom.close()


def test_edge_cases(lib):
    mesh = O.kuhn_box((3, 3, 3), 0.05)
    sp = O.plasma_species(1e10, 1.0, 1.0, 0.05, 2)
    dom = gpu_domain(mesh, 2e-8, face_bc=(1,) * 6)
    dom.set_species(sp)
    # empty species, one particle outside the mesh (lost at start -> absorbed at XMax)
    dom.set_particles(0, np.zeros((0, 3)), np.zeros((0, 3)))
    dom.set_particles(1, np.array([[0.2, 0.05, 0.05]]), np.array([[1.0, 0.0, 0.0]]))
    dom.set_potential(mesh.phi_bc)
    dom.step(2)
    p = dom.get_particles(1)
    assert p["status"][0] == O.ABSORBED and dom.ledger()[1, 5] == 1
    assert dom.count(0) == 0
    with pytest.raises(Exception):
        dom.set_particles(5, np.zeros((1, 3)), np.zeros((1, 3)))
    # a species re-sort interval needs a context interval to be a multiple of
    with pytest.raises(Exception):
        dom.set_species_sort_interval(1, 4)
    with pytest.raises(Exception):
        dom.set_species_sort_interval(7, 0)
    dom.set_species_sort_interval(1, 0)
    dom.close()
    dom = gpu_domain(mesh, 2e-8, face_bc=(1,) * 6, sort_interval=2)
    dom.set_species(sp)
    with pytest.raises(Exception):
        dom.set_species_sort_interval(1, 3)
    dom.set_species_sort_interval(1, 6)
    dom.close()


@pytest.mark.parametrize("precision", (0, 1))
def test_deterministic_and_sort_invariant(lib, precision):
    """Both forms give bitwise the same charge, potential, field, particles and ledger whatever
    the particle order: the re-sort moves state without arithmetic, the deposit and the push
    statistics are exact integer sums, and the PCG reductions have a fixed shape."""
    mesh = O.kuhn_box((8, 8, 8), 0.05, body=((3, 5), (3, 5), (3, 5)), bias=-10.0)
    sp = O.plasma_species(1e10, 1.0, 1.0, 0.05, 6)
    parts = O.seed_particles(mesh, sp, 6, 99)
    out = []
    # (re-sort interval, ion re-sort interval): none twice, every step, ions every third step
    for sort_interval, ion_interval in ((0, 0), (0, 0), (1, 0), (1, 3)):
        dom = gpu_domain(mesh, 2e-8, face_bc=(2, 2, 2, 2, 1, 1), precision=precision, sort_interval=sort_interval)
        gpu_load_particles(dom, sp, parts)
        if ion_interval:
            dom.set_species_sort_interval(1, ion_interval)
        dom.set_potential(mesh.phi_bc)
        dom.solve_field()
        dom.step(4)
        rho, phi, E = dom.fields()
        st = gpu_state(dom, len(sp), len(parts["tet"]))
        out.append((rho, phi, E, st, dom.ledger(), dom.stats()))
        dom.close()
    for k in (1, 2, 3):
        assert np.array_equal(out[0][0], out[k][0])  # fixed-point deposit: bitwise
        assert np.array_equal(out[0][1], out[k][1]) and np.array_equal(out[0][2], out[k][2])
        assert np.array_equal(out[0][4], out[k][4])
        act = out[0][3]["status"] == O.ACTIVE
        assert np.array_equal(out[0][3]["x"][act], out[k][3]["x"][act])
        for key in ("active_particles", "total_charge"):
            assert out[0][5][key] == out[k][5][key], key
    assert np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][2], out[1][2])
    # the kinetic energy is an integer sum, the same whichever warp took which particles (a
    # re-sort drops the inactive particles whose energy the statistics still count, so it is
    # compared between the two unsorted runs)
    assert out[0][5]["total_energy"] == out[1][5]["total_energy"]


def test_resort_gather_in_push_matches_gather_on_read(lib):
    """The precision form's re-sort leaves its gather to the next pass 1, which reads the store
    through the permutation; a read of the store in between (here the particles, every step)
    gathers it at once instead.  Both orders give bitwise the same run, with the stay-first ion
    pass and the walking pass both reading through a pending re-sort."""
    from scdat_b200 import capi

    mesh = O.kuhn_box((8, 8, 8), 0.05, body=((3, 5), (3, 5), (3, 5)), bias=-10.0)
    sp = O.plasma_species(1e10, 1.0, 1.0, 0.05, 6)
    parts = O.seed_particles(mesh, sp, 6, 7)
    out = []
    for read_between, ion_mode in ((False, capi.PUSH_STAY_FIRST), (True, capi.PUSH_STAY_FIRST),
                                   (False, capi.PUSH_WALKING)):
        dom = gpu_domain(mesh, 2e-8, face_bc=(2, 2, 2, 2, 1, 1), precision=1, sort_interval=1)
        gpu_load_particles(dom, sp, parts)
        dom.set_push_mode(1, ion_mode)
        dom.set_potential(mesh.phi_bc)
        dom.solve_field()
        for _ in range(5):
            dom.step(1)
            if read_between:
                gpu_state(dom, len(sp), len(parts["tet"]))
        dom.compact()  # a re-sort with no push after it: read back through the gather
        rho, phi, E = dom.fields()
        out.append((rho, phi, gpu_state(dom, len(sp), len(parts["tet"])), dom.ledger(), dom.stats()))
        dom.close()
    for k in (1, 2):
        assert np.array_equal(out[0][0], out[k][0]) and np.array_equal(out[0][1], out[k][1])
        for key in ("x", "v", "tet", "status"):
            assert np.array_equal(out[0][2][key], out[k][2][key], equal_nan=True), key
        assert np.array_equal(out[0][3], out[k][3])
        assert out[0][4]["total_energy"] == out[k][4]["total_energy"]


def test_mixed_precision_error_bounded(lib):
    """Precision form against the FP64 form on the same inputs (errors reported and bounded)."""
    mesh, sp, parts, dt, nsteps, face_bc = make_inputs("box6_body")
    res = {}
    for prec in (0, 1):
        dom = gpu_domain(mesh, dt, face_bc=face_bc, precision=prec, pcg_rtol=1e-10)
        gpu_load_particles(dom, sp, parts)
        dom.set_potential(mesh.phi_bc)
        dom.solve_field()
        dom.step(3)
        res[prec] = (dom.fields(), gpu_state(dom, len(sp), len(parts["tet"])))
        dom.close()
    (r0, p0, e0), s0 = res[0]
    (r1, p1, e1), s1 = res[1]
    assert rel_err(p1, p0) < 1e-6
    assert rel_err(e1, e0) < 1e-4
    both = (s0["status"] == O.ACTIVE) & (s1["status"] == O.ACTIVE)
    assert (s0["status"] != s1["status"]).mean() < 0.005
    assert both.sum() > 0.9 * (s0["status"] == O.ACTIVE).sum()
    assert np.abs(s1["x"][both] - s0["x"][both]).max() < 1e-6


def test_stay_first_push_is_bitwise_the_walking_push(lib):
    """The precision form's stay-first pass 1 (no walk code; particles leaving their tet go to
    the walking passes, which redo that sub-step) against the walking pass 1, for both species,
    over steps with re-sorts, MCC and particles lost at the faces: charge, potential, field,
    particles, ledger and statistics bitwise equal; the automatic choice likewise."""
    from scdat_b200 import capi

    mesh = O.kuhn_box((10, 9, 8), 0.05, body=((4, 6), (3, 6), (3, 5)), bias=-30.0)
    sp = O.plasma_species(1e10, 2.0, 1.0, 0.05, 6)
    parts = O.seed_particles(mesh, sp, 6, 123)
    out = []
    for mode in (capi.PUSH_WALKING, capi.PUSH_STAY_FIRST, capi.PUSH_AUTO):
        dom = gpu_domain(mesh, 3e-8, face_bc=(2, 2, 1, 1, 1, 1), precision=1, sort_interval=2, seed=9)
        gpu_load_particles(dom, sp, parts)
        for s in range(len(sp)):
            dom.set_push_mode(s, mode)
            dom.set_elastic(s, 3e19, 1e-19)
        dom.set_potential(mesh.phi_bc)
        dom.solve_field()
        dom.step(6)
        rho, phi, E = dom.fields()
        st = gpu_state(dom, len(sp), len(parts["tet"]))
        out.append((rho, phi, E, st, dom.ledger(), dom.stats()))
        dom.close()
    ref = out[0]
    assert ref[4][:6, 4:6].sum() > 0 and ref[5]["mcc_collisions"] > 0
    for k in (1, 2):
        for j in (0, 1, 2, 4):
            assert np.array_equal(out[k][j], ref[j]), (k, j)
        for key in ("x", "v", "tet", "status"):
            assert np.array_equal(np.nan_to_num(out[k][3][key]), np.nan_to_num(ref[3][key])), (k, key)
        for key in ("active_particles", "total_charge", "total_energy", "substeps", "lost_events", "mcc_collisions"):
            assert out[k][5][key] == ref[5][key], (k, key)
