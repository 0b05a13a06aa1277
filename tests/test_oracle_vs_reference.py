"""Pin the C oracle against the reference's own classes, compiled from its sources into
oracle/_ref (skipped where that library was not built), on identical seeded state."""
import numpy as np
import pytest

import oracle as O
from conftest import rel_err
from golden.make_golden import CASES
from pic_helpers import oracle_cycle, oracle_mcc_run


def _setup(n=(5, 5, 5), body=((2, 3), (2, 3), (2, 3)), bias=-10.0, ppc=3, seed=5):
    mesh = O.kuhn_box(n, 0.05, body=body, bias=bias)
    sp = O.plasma_species(1e10, 1.0, 1.0, 0.05, ppc)
    parts = O.seed_particles(mesh, sp, ppc, seed)
    return mesh, sp, parts


def test_philox_known_answers(orc):
    # Random123 known-answer vectors for Philox4x32-10
    assert list(orc.philox([0, 0, 0, 0], [0, 0])) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert list(orc.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert list(orc.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0])) == [
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]
    ctr = np.array([[1, 2, 3, 4], [0, 0, 0, 0]], np.uint32)
    key = np.array([[5, 6], [0, 0]], np.uint32)
    vec = O.philox4x32_10(ctr, key)
    assert list(vec[1]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert list(vec[0]) == list(orc.philox([1, 2, 3, 4], [5, 6]))


def test_boris_known_answer(orc):
    # Tools/Particle/test/ParticleDefinitions_test.cpp:72-91: q/m = 1, E = 2 x, dt = 0.5 -> v = 1
    out = np.zeros(3)
    orc.L.orc_boris(np.zeros(3), np.array([2.0, 0.0, 0.0]), 1.0, 0.5, out)
    assert abs(out[0] - 1.0) < 1e-12 and out[1] == 0.0 and out[2] == 0.0


@pytest.mark.parametrize("neighbors", [True, False])
@pytest.mark.parametrize("kernel", [0, 1, 2])
def test_push_variants(orc, ref, neighbors, kernel):
    mesh, sp, parts = _setup()
    phi, E = ref.poisson(mesh, np.zeros(mesh.N), mesh.phi_bc)
    a = orc.push(mesh, E, parts, sp, 3e-8, kernel=kernel, neighbors=neighbors)
    b = ref.push(mesh, E, parts, sp, 3e-8, kernel=kernel, neighbors=neighbors)
    assert np.array_equal(a["tet"], b["tet"]) and np.array_equal(a["lost"], b["lost"])
    assert a["substeps"] == b["substeps"]
    assert rel_err(a["x"], b["x"]) < 1e-12
    assert rel_err(a["v"], b["v"]) < 1e-12
    assert rel_err(a["rho"], b["rho"]) < 1e-12


def test_push_without_hints(orc, ref):
    # no location hints: the reference falls back to its linear scan (lowest containing id)
    mesh, sp, parts = _setup(n=(4, 4, 4), body=None, ppc=2)
    parts = dict(parts, tet=np.full_like(parts["tet"], -1))
    E = np.zeros((mesh.N, 3))
    a = orc.push(mesh, E, parts, sp, 2e-8)
    b = ref.push(mesh, E, parts, sp, 2e-8)
    assert np.array_equal(a["tet"], b["tet"]) and rel_err(a["rho"], b["rho"]) < 1e-12


def test_lsq_set_potential(orc, ref):
    # PICCycle::setPotential -> updateElectricField (PICCycle.cpp:769-894), 1e-18 regularisation
    mesh, _, _ = _setup(body=None)
    phi = 12.0 * mesh.xyz[:, 2] + 3.0 * mesh.xyz[:, 0] ** 2
    A = orc.assemble(mesh)
    assert rel_err(orc.lsq(mesh, A, phi, reg=1e-18), ref.lsq(mesh, phi)) < 1e-12


def test_poisson_plate_reference_test(orc, ref):
    # Tools/FieldSolver/test/PoissonSolver_test.cpp:48-117: 10 V / 0 V plates, interior in [0,10]
    mesh = O.kuhn_box((1, 1, 6), 0.01, body=None)
    z = mesh.xyz[:, 2]
    dir_ = ((z < 1e-12) | (z > z.max() - 1e-12)).astype(np.uint8)
    phi_bc = np.where(z < 1e-12, 10.0, 0.0)
    mesh.dirichlet[:] = dir_
    mesh.phi_bc[:] = phi_bc
    A = orc.assemble(mesh)
    phi, _, _ = orc.poisson(mesh, A, np.zeros(mesh.N), phi_bc)
    inner = dir_ == 0
    assert np.all(phi[inner] >= -1e-8) and np.all(phi[inner] <= 10 + 1e-8)
    assert np.allclose(phi[z < 1e-12], 10.0, atol=1e-8)
    pr, Er = ref.poisson(mesh, np.zeros(mesh.N), phi_bc)
    assert rel_err(phi, pr) < 1e-12
    E = orc.lsq(mesh, A, phi)
    assert np.all(np.isfinite(E)) and np.abs(E).max() > 0 and rel_err(E, Er) < 1e-12


@pytest.mark.parametrize("face_bc", [(2, 2, 2, 2, 1, 1), (1, 1, 1, 1, 1, 1), (0, 0, 0, 0, 1, 1)])
def test_cycle_boundaries(orc, ref, face_bc):
    mesh, sp, parts = _setup(ppc=3)
    phi0, _ = ref.poisson(mesh, np.zeros(mesh.N), mesh.phi_bc)
    a = oracle_cycle(orc, mesh, sp, parts, 3, 4e-8, face_bc, phi0)
    b = ref.cycle(mesh, parts, sp, 3, 4e-8, face_bc, phi0)
    ids = b["id"]
    st = {10: O.ACTIVE, 20: O.ABSORBED, 21: O.ESCAPED}
    assert np.array_equal(a["status"][ids], np.array([st[s] for s in b["status"]]))
    act = b["status"] == 10
    assert rel_err(a["x"][ids][act], b["x"][act]) < 1e-12
    assert rel_err(a["rho"], b["rho"]) < 1e-12
    assert rel_err(a["phi"], b["phi"]) < 1e-12
    np.testing.assert_allclose(a["ledger"][:6], b["ledger"], rtol=1e-12, atol=1e-30)


def _plate():
    # the 1 x 1 x 6 plate of Tools/PICcore/test/PICCycleBoundary_test.cpp:32-65 (Kuhn split)
    mesh = O.kuhn_box((1, 1, 6), 1.0 / 1.0, body=None)
    mesh.xyz[:, 2] /= 6.0
    z = mesh.xyz[:, 2]
    mesh.dirichlet[:] = ((z < 1e-12) | (z > z.max() - 1e-12)).astype(np.uint8)
    mesh.phi_bc[:] = 0.0
    return mesh


def _single(mesh, tet, vel, w=1.0):
    c = mesh.xyz[mesh.tet[tet]].mean(axis=0)
    return dict(x=c[None, :].copy(), v=np.array([vel], np.float64), species=np.zeros(1, np.int32),
                tet=np.array([tet], np.int32), id=np.zeros(1, np.int64))


@pytest.mark.parametrize("scenario", ["periodic", "absorbing", "far_escape"])
def test_picycle_boundary_reference_tests(orc, ref, scenario):
    """PICCycleBoundary_test.cpp:121-221 re-hosted: dt 1e-9, one electron of weight 1."""
    mesh = _plate()
    sp = [O.Species(-O.QE, O.ME, 1.0, 0, 1.0)]
    cent = mesh.xyz[mesh.tet].mean(axis=1)
    if scenario == "periodic":
        t = int(np.argmax(cent[:, 0]))
        parts, bc = _single(mesh, t, [2.0e9, 0, 0]), (2, 2, 2, 2, 1, 1)
    elif scenario == "absorbing":
        t = int(np.argmax(cent[:, 2]))
        parts, bc = _single(mesh, t, [0, 0, 2.0e9]), (2, 2, 2, 2, 1, 1)
    else:
        t = int(np.argmax(cent[:, 2]))
        parts, bc = _single(mesh, t, [0, 0, 5.0e12]), (0, 0, 0, 0, 0, 0)
    phi0 = np.zeros(mesh.N)
    a = oracle_cycle(orc, mesh, sp, parts, 1, 1e-9, bc, phi0)
    b = ref.cycle(mesh, parts, sp, 1, 1e-9, bc, phi0)
    st = {10: O.ACTIVE, 20: O.ABSORBED, 21: O.ESCAPED}
    assert a["status"][0] == st[b["status"][0]]
    if scenario == "periodic":
        assert a["status"][0] == O.ACTIVE
        assert -1e-9 <= a["x"][0, 0] <= 1.0 + 1e-9
        assert rel_err(a["x"], b["x"]) < 1e-12
    elif scenario == "absorbing":
        assert a["status"][0] == O.ABSORBED
        assert a["surface_charge"] < 0 and a["ledger"][5, 0] < 0 and a["ledger"][5, 4] == 1
        np.testing.assert_allclose(a["ledger"][:6], b["ledger"], rtol=1e-12, atol=1e-40)
    else:
        assert a["status"][0] != O.ACTIVE and abs(a["surface_charge"]) < 1e-20


def test_mcc_statistics_match_reference(orc, ref):
    """Reference mt19937 stream vs oracle Philox streams: the same collision law within a
    5-sigma band (the streams themselves cannot match).  The reference handler counts
    first-draw hits (probability p) while a particle scatters only when its second draw
    passes too (probability p^2)."""
    rng = np.random.default_rng(3)
    P = 20000
    v = rng.normal(size=(P, 3)) * 4.2e5
    sigma, n_t, dt, reps = 1e-19, 3e20, 2e-8, 5
    ref_hits, ref_scat = ref.mcc_count(v, 0, 1.0, sigma, n_t, dt, 7, reps)
    sp = [O.Species(-O.QE, O.ME, 1.0, 0, 1.0)]
    proc = [O.Elastic(n_t, sigma, 1.0, 0.0, 0.0, 1, 0)]
    hits = 0
    for r in range(reps):
        _, h = orc.mcc(v, np.zeros(P, np.int32), np.zeros(P, np.uint8), np.arange(P), sp, proc, dt, 99, r, mode=0)
        hits += h
    p = np.clip(n_t * sigma * np.linalg.norm(v, axis=1) * dt, 0, 1)
    m1, s1 = reps * p.sum(), np.sqrt(reps * np.sum(p * (1 - p)))
    m2, s2 = reps * np.sum(p * p), np.sqrt(reps * np.sum(p * p * (1 - p * p)))
    assert abs(ref_hits - m1) < 5 * s1, (ref_hits, m1, s1)
    assert abs(ref_scat - m2) < 5 * s2, (ref_scat, m2, s2)
    assert abs(hits - m2) < 5 * s2, (hits, m2, s2)


def test_full_mcc_run_matches_reference_statistically(orc, ref):
    """A full PIC-MCC run of the reference (PICCycle steps, each followed by its background MCC
    step on one mt19937 stream) against the oracle's run on Philox streams, from the same
    particles.  The streams cannot match, so the runs are compared statistically: per species
    the mean x-velocity, the mean squared speed and the surviving count, and per face the
    collected electron and ion counts, each within 5 sigma of the difference (the sampling
    errors of the two runs added as if independent, which overstates them since the runs
    share their initial state).  Electrons start with a +x drift of two thermal speeds and
    collide often, so the drift left after the run measures the collisions: without MCC it
    lies far outside the band.  The floating potential is not on this reference path (the
    reference's PICCycle has no surface circuit), so it is not compared here."""
    mesh = O.kuhn_box((6, 6, 6), 0.05)
    ppc, nsteps, dt, sigma, n_t = 40, 8, 2e-8, 1e-19, 3e20
    sp = O.plasma_species(1e10, 1.0, 1.0, 0.05, ppc)
    parts = O.seed_particles(mesh, sp, ppc, 100)
    vth = np.sqrt(O.QE / O.ME)
    parts["v"][parts["species"] == 0, 0] += 2.0 * vth
    face_bc = (1,) * 6
    run = oracle_mcc_run(orc, mesh, sp, parts, nsteps, dt, face_bc, n_t, sigma, 1000)
    mine, led = run["parts"], run["ledger"]
    theirs = ref.cycle_mcc(mesh, parts, sp, nsteps, dt, face_bc, mesh.phi_bc, n_t, sigma, 2000)
    their_species = parts["species"][theirs["id"]]

    def z_means(a, b):
        return abs(a.mean() - b.mean()) / np.sqrt(a.var() / len(a) + b.var() / len(b))

    for s in (0, 1):
        a, b = mine["v"][mine["species"] == s], theirs["v"][their_species == s]
        assert len(a) > 1000 and len(b) > 1000
        assert z_means(a[:, 0], b[:, 0]) < 5.0, ("mean vx", s)
        assert z_means((a ** 2).sum(1), (b ** 2).sum(1)) < 5.0, ("mean v^2", s)
        assert abs(len(a) - len(b)) < 5.0 * np.sqrt(len(a) + len(b)), ("survivors", s)
    for f in range(6):
        for col in (4, 5):  # absorbed electron and ion macro-particles on face f
            c1, c2 = led[f, col], theirs["ledger"][f, col]
            assert abs(c1 - c2) < 5.0 * np.sqrt(c1 + c2 + 1.0), (f, col, c1, c2)
    assert theirs["ledger"][1, 4] > 100  # the drift carries electrons to the +x face

    # power: the same run without collisions keeps most of the drift
    free = oracle_mcc_run(orc, mesh, sp, parts, nsteps, dt, face_bc, 0.0, sigma, 1000)["parts"]
    a = free["v"][free["species"] == 0][:, 0]
    b = theirs["v"][their_species == 0][:, 0]
    assert z_means(a, b) > 10.0


def test_surface_circuit_matches_reference(ref):
    """The oracle's face-potential update (the device's rule) against the reference's
    SurfaceCircuitCoupling::advanceImplicit on random independent nodes: capacitances of
    dielectric patches, shunt conductances, plasma currents and their linearisation."""
    rng = np.random.default_rng(17)
    mesh = O.kuhn_box((4, 4, 4), 0.05, body=((1, 3), (1, 3), (1, 3)), bias=0.0)
    for trial in range(200):
        sc = O.SurfaceCircuit(mesh, (0.05, 0.05, 0.05), (0.15, 0.15, 0.15), eps_r=rng.uniform(1, 10),
                              thickness=10 ** rng.uniform(-5, -2))
        sc.C = sc.C * rng.uniform(0.5, 2.0, 6)
        sc.G = np.where(rng.random(6) < 0.5, 0.0, 10 ** rng.uniform(-12, -6, 6))
        sc.didv = np.where(rng.random(6) < 0.3, 0.0, -(10 ** rng.uniform(-12, -6, 6)))
        sc.V = rng.uniform(-1000.0, 100.0, 6)
        dt = 10 ** rng.uniform(-10, -7)
        dq = rng.normal(0.0, 1e-12, 6)
        V0, C0, G0, D0 = sc.V.copy(), sc.C.copy(), sc.G.copy(), sc.didv.copy()
        sc.advance(dq, dt)
        theirs = ref.circuit_advance(C0, G0, V0, dq / dt, D0, dt)
        np.testing.assert_allclose(sc.V, theirs, rtol=1e-12, atol=1e-12 * np.abs(V0).max())


def test_whipple_yield_matches_reference(ref):
    """The oracle's (and the device's) Whipple secondary yield against the reference's
    evaluateLegacySecondaryElectronYield, over incident energies from 0 to 20 keV and several
    peak yields and peak energies (including a peak energy below the reference's 1 eV floor)."""
    e = np.concatenate([[0.0, 1e-6, 0.5], np.geomspace(1e-3, 1.0, 40), np.linspace(1.0, 2e4, 400)])
    for peak_yield in (0.0, 0.7, 2.0, 3.5):
        for peak_e in (0.3, 50.0, 300.0, 800.0):
            mine = O.see_yield(2, peak_yield, peak_e, e)
            theirs = ref.whipple_yield(peak_yield, peak_e, e)
            # q = 2.28 (E/Emax)^1.35; the numerator q - 1 + exp(-q) ~ q^2/2 cancels for small q,
            # so an ulp of exp or pow grows by ~2/q^2 there: the bar is 1e-12 or that condition
            # number times a few ulps, whichever is larger
            q = 2.28 * (e / max(1.0, peak_e)) ** 1.35
            bar = np.maximum(1e-12, 1e-15 / np.maximum(q * q / 2.0, 1e-300))
            assert np.all(np.abs(mine - theirs) <= bar * np.abs(theirs)), (peak_yield, peak_e)
            assert np.all(bar[e >= 0.1 * max(1.0, peak_e)] < 1e-12 * 1.5)  # the plain bar above 0.1 Emax


def test_null_collision_law(orc):
    """Null-collision MCC (mode 2) against the direct draw (mode 1) on 400k Maxwellian
    electrons at nu dt ~ 1e-2: each mode's collision count within 5 sigma of its own expected
    value (sum of the per-particle probabilities: 1 - exp(-nu dt), and
    (1 - exp(-nu_max dt)) nu / nu_max), the two laws equal to first order in nu dt, speeds kept;
    particles faster than the bound take the direct draw."""
    rng = np.random.default_rng(8)
    n = 400_000
    sp = [O.Species(-O.QE, O.ME, 1.0, 0, 1.0)]
    v = rng.normal(0.0, np.sqrt(O.QE / O.ME), (n, 3))
    spd = np.linalg.norm(v, axis=1)
    idx = np.zeros(n, np.int32)
    status = np.zeros(n, np.uint8)
    ids = np.arange(n, dtype=np.int64)
    n_t, sigma, dt = 4e19, 1e-19, 4e-9
    proc = [O.Elastic(n_t, sigma, 1.0, 0.0, 0.0, 1, 0)]
    nu = n_t * sigma * spd
    for vbound in (spd.max(), np.quantile(spd, 0.9)):
        numax = n_t * sigma * vbound
        slow = spd <= vbound
        p2 = np.where(slow, (1.0 - np.exp(-numax * dt)) * nu / numax, 1.0 - np.exp(-nu * dt))
        p1 = 1.0 - np.exp(-nu * dt)
        for mode, p in ((1, p1), (2, p2)):
            v2, hits = orc.mcc(v, idx, status, ids, sp, proc, dt, 77, 3, mode=mode, vmax=np.array([vbound]))
            mu, sd = p.sum(), np.sqrt((p * (1 - p)).sum())
            assert abs(hits - mu) < 5 * sd, (mode, vbound, hits, mu, sd)
            np.testing.assert_allclose(np.linalg.norm(v2, axis=1), spd, rtol=1e-12)
            assert np.count_nonzero(np.any(v2 != v, axis=1)) == hits
        assert abs(p2.sum() - p1.sum()) < 0.02 * p1.sum()  # same law to O(nu dt)
    # the two modes draw from different streams, so their collision sets differ
    _, h1 = orc.mcc(v, idx, status, ids, sp, proc, dt, 77, 3, mode=1)
    assert h1 > 1000


def test_csv_export_matches_reference_exporter(ref, tmp_path):
    """scdat_export_columns_csv against the reference's own CSVExporter::exportDataSet
    (Tools/Output/src/CSVExporter.cpp:11-47) on the same columnar data: byte-identical files,
    series in name order, the parent directories created, signed zeros, extreme exponents and
    non-finite values written alike; a repeated name keeps its last series, as std::map does."""
    from scdat_b200 import build, capi

    build.build()  # host code: runs without a GPU
    rng = np.random.default_rng(11)
    n = 57
    axis = np.linspace(-0.5, 1.25, n)
    series = {"potential_v": rng.normal(0.0, 3.0, n), "electron_density_m3": 10 ** rng.uniform(6, 18, n),
              "Z_upper": rng.normal(0.0, 1e-300, n), "a_first": rng.uniform(-1, 1, n) * 1e300,
              "electric_field_z_v_per_m": rng.normal(0.0, 1e3, n)}
    series["potential_v"][[0, 3, 5]] = [-0.0, np.inf, np.nan]
    series["a_first"][7] = -np.inf
    for k, (name, vals) in enumerate([("index", series), ("z_m", {"only": axis * 2.0}), ("node", {})]):
        ours, theirs = tmp_path / f"ours{k}" / "sub" / "t.csv", tmp_path / f"ref{k}" / "sub" / "t.csv"
        capi.export_columns_csv(ours, name, axis, vals)
        assert ref.csv_export(theirs, name, axis, vals)
        assert ours.read_bytes() == theirs.read_bytes()
    # a repeated name: ours is given the pair list, the reference's map keeps the last assignment
    L = capi.load()
    import ctypes as C

    a = np.ascontiguousarray(axis)
    v1, v2 = np.ones(n), np.full(n, 2.0)
    names = (C.c_char_p * 2)(b"dup", b"dup")
    vals = (C.c_void_p * 2)(v1.ctypes.data, v2.ctypes.data)
    assert L.scdat_export_columns_csv(str(tmp_path / "dup.csv").encode(), b"x", n, a.ctypes.data, 2, names, vals) == 0
    assert ref.csv_export(tmp_path / "dup_ref.csv", "x", axis, {"dup": v2})
    assert (tmp_path / "dup.csv").read_bytes() == (tmp_path / "dup_ref.csv").read_bytes()


@pytest.mark.parametrize("model", ["sims", "katz"])
def test_legacy_sims_katz_yields_match_reference(ref, model):
    """The oracle's (and the device's) Sims and Katz secondary yields against the reference's
    evaluateLegacySecondaryElectronYield over 0-20 keV, several peak yields and energies, and
    several Sims exponents (below the 1.05 floor too) and Katz range coefficients."""
    e = np.concatenate([[0.0, 1e-12, 1e-9, 0.5, 9.999, 10.0, 10.001], np.geomspace(1e-3, 50.0, 60),
                        np.linspace(50.0, 2e4, 400)])
    shapes = [dict(sims_n=n) for n in (0.9, 1.05, 1.35, 1.6, 2.2)] if model == "sims" else \
        [dict(katz=k) for k in ((0.85, 0.35, 0.12, 1.05), (1.2, 0.5, 0.05, 1.4), (0.4, 0.2, 0.3, 0.9))]
    num = 3 if model == "sims" else 4
    for peak_yield in (0.0, 0.7, 2.0, 3.5):
        for peak_e in (0.3, 50.0, 300.0, 800.0):
            for sh in shapes:
                mine = O.see_yield(num, peak_yield, peak_e, e, **sh)
                theirs = ref.legacy_yield(model, peak_yield, peak_e, e, **sh)
                assert np.array_equal(mine == 0.0, theirs == 0.0), (peak_yield, peak_e, sh)
                if model == "sims":
                    # the numerator x + e^-x - 1 ~ x^2/2 cancels for small x = xm (E/Emax)^n, so
                    # an ulp of exp grows by ~2/x^2: the bar is 1e-12 or that condition number
                    # times a few ulps, whichever is larger
                    n = max(1.05, sh["sims_n"])
                    x = O.sims_xm(n) * (e / max(1.0, peak_e)) ** n
                    bar = np.maximum(1e-12, 1e-15 * 2.0 / np.maximum(x * x, 1e-300))
                else:
                    bar = np.full_like(e, 1e-12)
                assert np.all(np.abs(mine - theirs) <= bar * np.abs(theirs)), (peak_yield, peak_e, sh)


def test_sampler_fixture_is_the_reference_sampler(ref):
    """tests/golden/sampler_ref.npz (the GPU sampler test's reference) is what the reference's
    PicMccSurfaceCurrentSampler gives here: its plate mesh and its sampleWithDerivative output
    at both potentials, reproduced exactly from the recorded configuration and seed."""
    import os

    from golden.make_golden import SAMPLER, SAMPLER_POTENTIALS

    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sampler_ref.npz"))
    c = SAMPLER
    xyz, tet = ref.sampler_mesh(c["area_m2"], c["aspect"], c["gap_m"], c["z_layers"])
    assert np.array_equal(xyz, g["xyz"]) and np.array_equal(tet, g["tet"])
    assert np.array_equal(g["potentials"], np.array(SAMPLER_POTENTIALS))
    for v, row in zip(SAMPLER_POTENTIALS, g["samples"]):
        out = ref.sampler_sample(c["area_m2"], c["gap_m"], c["z_layers"], c["ppe"], c["window_steps"], c["seed"],
                                 c["ne"], c["ni"], c["te_ev"], c["ti_ev"], c["ion_amu"], v, c["reference_v"],
                                 c["probe_dv"])
        assert out["valid"] == 1.0
        got = [out[k] for k in ("electron", "ion", "emitted", "net", "derivative", "segments")]
        assert np.array_equal(np.array(got), row), v


@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_fixtures_are_the_reference(ref, name):
    """Each small-case fixture in tests/golden (the GPU parity tests' reference values) is what
    the reference's own code gives here from the recorded inputs: Laplace solve, frozen-field
    push, charged solve and the full cycle, reproduced exactly."""
    import os

    from golden.make_golden import make_inputs

    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", f"{name}.npz"))
    mesh, sp, parts, dt, nsteps, face_bc = make_inputs(name)
    phi_l, E_l = ref.poisson(mesh, np.zeros(mesh.N), mesh.phi_bc)
    push = ref.push(mesh, E_l, parts, sp, dt)
    phi_q, E_q = ref.poisson(mesh, push["rho"], mesh.phi_bc)
    cyc = ref.cycle(mesh, parts, sp, nsteps, dt, face_bc, phi_l)
    pairs = {"phi_laplace": phi_l, "E_laplace": E_l, "push_x": push["x"], "push_v": push["v"],
             "push_tet": push["tet"], "push_lost": push["lost"], "push_rho": push["rho"],
             "push_substeps": push["substeps"], "phi_charge": phi_q, "E_charge": E_q, "cyc_x": cyc["x"],
             "cyc_v": cyc["v"], "cyc_id": cyc["id"], "cyc_status": cyc["status"], "cyc_rho": cyc["rho"],
             "cyc_phi": cyc["phi"], "cyc_E": cyc["E"], "cyc_ledger": cyc["ledger"], "cyc_stats": cyc["stats"]}
    for key, val in pairs.items():
        assert np.array_equal(np.asarray(val), g[key], equal_nan=True), key


def test_config0_fixture_is_the_reference(ref):
    """tests/golden/config0_ref.npz is the reference's push of the first benchmark
    configuration's subsample in the reference's LSQ field of the Laplace potential, reproduced
    exactly here from the recorded inputs."""
    import os

    from golden.make_golden import CONFIG0_STRIDE, config0_laplace, make_config0_inputs, subsample

    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "config0_ref.npz"))
    mesh, sp, parts, dt = make_config0_inputs()
    o = O.Oracle(fast_locate=True)
    try:
        _, phi = config0_laplace(o, mesh)
    finally:
        o.close()
    E = ref.lsq(mesh, phi)
    push = ref.push(mesh, E, subsample(parts, CONFIG0_STRIDE), sp, dt)
    nz = np.nonzero(push["rho"])[0]
    assert g["phi_sum"] == np.sum(phi) and g["E_abs_sum"] == np.sum(np.abs(E))
    for key in ("x", "v", "tet", "lost", "substeps"):
        assert np.array_equal(np.asarray(push[key]), g["push_" + key]), key
    assert np.array_equal(nz, g["rho_nodes"]) and np.array_equal(push["rho"][nz], g["rho_vals"])


def test_push_edge_cases_match_reference(orc, ref):
    """Edge inputs through both the oracle and the reference's CrossTetrahedron: no particles
    (no charge, no sub-steps), a particle outside the mesh with no location hint (lost at once,
    state untouched, nothing deposited), and one exactly on a shared vertex of the box."""
    mesh = O.kuhn_box((3, 3, 3), 0.05)
    sp = O.plasma_species(1e10, 1.0, 1.0, 0.05, 2)
    E = np.zeros((mesh.N, 3))

    def parts(x, v, s, t):
        return dict(x=np.asarray(x, float).reshape(-1, 3), v=np.asarray(v, float).reshape(-1, 3),
                    species=np.asarray(s, np.int32), tet=np.asarray(t, np.int32),
                    id=np.arange(len(s), dtype=np.int64))

    cases = [parts([], [], [], []),
             parts([[0.2, 0.05, 0.05]], [[1.0, 0.0, 0.0]], [1], [-1]),
             parts([[0.05, 0.05, 0.05]], [[10.0, -5.0, 2.0]], [0], [-1])]
    for p in cases:
        a, b = orc.push(mesh, E, p, sp, 2e-8), ref.push(mesh, E, p, sp, 2e-8)
        assert np.array_equal(a["lost"], b["lost"]) and np.array_equal(a["tet"], b["tet"])
        assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["v"], b["v"])
        assert np.abs(a["rho"] - b["rho"]).max(initial=0.0) <= 1e-12 * np.abs(b["rho"]).max(initial=1e-300)
        assert a["substeps"] == b["substeps"]
    assert np.abs(orc.push(mesh, E, cases[0], sp, 2e-8)["rho"]).max() == 0.0


@pytest.mark.parametrize("cells", [(1, 1, 1), (2, 2, 2), (2, 1, 3)])
def test_poisson_degenerate_meshes_match_reference(orc, ref, cells):
    """Meshes with no unknown (every node Dirichlet) or a single one: the oracle's solve and LSQ
    field against the reference's PoissonSolver and PICCycle field, with random boundary values
    and charge."""
    mesh = O.kuhn_box(cells, 0.05, bias=0.0)
    rng = np.random.default_rng(1)
    phi_bc = mesh.phi_bc + rng.normal(0.0, 1.0, mesh.N) * (mesh.dirichlet == 1)
    rho = rng.normal(0.0, 1e-12, mesh.N)
    A = orc.assemble(mesh)
    phi, _, _ = orc.poisson(mesh, A, rho, phi_bc)
    E = orc.lsq(mesh, A, phi)
    ref_phi, ref_E = ref.poisson(mesh, rho, phi_bc)
    assert np.abs(phi - ref_phi).max() <= 1e-12 * np.abs(ref_phi).max()
    assert rel_err(E, ref_E) < 1e-12
