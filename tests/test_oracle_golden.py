"""The C oracle against fixtures produced by the reference's own classes (tests/golden)."""
import os

import numpy as np
import pytest

import oracle as O
from pic_helpers import oracle_cycle
from golden.make_golden import CASES, make_inputs
from conftest import rel_err

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request):
    return request.param, np.load(os.path.join(GOLDEN, f"{request.param}.npz"))


def test_poisson_laplace(orc, case):
    name, g = case
    mesh, sp, parts, dt, nsteps, face_bc = make_inputs(name)
    A = orc.assemble(mesh)
    phi, it, rel = orc.poisson(mesh, A, np.zeros(mesh.N), mesh.phi_bc)
    assert rel < 1e-14
    assert rel_err(phi, g["phi_laplace"]) < 1e-12
    assert rel_err(orc.lsq(mesh, A, phi), g["E_laplace"]) < 1e-12


def test_push_frozen_field(orc, case):
    name, g = case
    mesh, sp, parts, dt, nsteps, face_bc = make_inputs(name)
    out = orc.push(mesh, g["E_laplace"], parts, sp, dt)
    assert np.array_equal(out["tet"], g["push_tet"])
    assert np.array_equal(out["lost"], g["push_lost"])
    assert out["substeps"] == int(g["push_substeps"])
    assert np.abs(out["x"] - g["push_x"]).max() < 1e-12 * np.abs(g["push_x"]).max()
    assert rel_err(out["v"], g["push_v"]) < 1e-12
    assert rel_err(out["rho"], g["push_rho"]) < 1e-12


def test_poisson_with_charge(orc, case):
    name, g = case
    mesh, *_ = make_inputs(name)
    A = orc.assemble(mesh)
    phi, _, _ = orc.poisson(mesh, A, g["push_rho"], mesh.phi_bc)
    assert rel_err(phi, g["phi_charge"]) < 1e-12
    assert rel_err(orc.lsq(mesh, A, phi), g["E_charge"]) < 1e-12


def test_full_cycle(orc, case):
    name, g = case
    mesh, sp, parts, dt, nsteps, face_bc = make_inputs(name)
    res = oracle_cycle(orc, mesh, sp, parts, nsteps, dt, face_bc, g["phi_laplace"])
    ids = g["cyc_id"]
    act = g["cyc_status"] == 10
    assert np.array_equal(res["status"][ids] == O.ACTIVE, act)
    assert np.array_equal(res["status"][ids] == O.ABSORBED, g["cyc_status"] == 20)
    assert np.abs(res["x"][ids][act] - g["cyc_x"][act]).max() < 1e-12 * np.abs(g["cyc_x"]).max()
    assert rel_err(res["v"][ids][act], g["cyc_v"][act]) < 1e-12
    assert rel_err(res["rho"], g["cyc_rho"]) < 1e-12
    assert rel_err(res["phi"], g["cyc_phi"]) < 1e-12
    assert rel_err(res["E"], g["cyc_E"]) < 1e-12
    led = g["cyc_ledger"]
    assert np.array_equal(res["ledger"][:6, 4:6], led[:, 4:6])
    np.testing.assert_allclose(res["ledger"][:6, :4], led[:, :4], rtol=1e-12, atol=1e-30)
    np.testing.assert_allclose(res["surface_charge"], g["cyc_stats"][4], rtol=1e-12, atol=1e-30)


def test_fast_locate_is_the_linear_scan(orc):
    """The oracle's scan accelerator returns the lowest-id containing tet for every point, as
    the linear scan: random points (inside, in the body hole, outside), points on shared faces,
    edges and vertices, and full pushes with and without neighbour lists."""
    fast = O.Oracle(fast_locate=True)
    mesh = O.kuhn_box((6, 5, 4), 0.05, body=((2, 4), (1, 3), (1, 3)), bias=-10.0)
    rng = np.random.default_rng(11)
    lo, hi = mesh.xyz.min(axis=0), mesh.xyz.max(axis=0)
    pts = [lo - 0.02 + rng.random(3) * (hi - lo + 0.04) for _ in range(3000)]
    pts += [mesh.xyz[i] for i in rng.integers(0, mesh.N, 300)]  # vertices
    tn = mesh.tet[rng.integers(0, mesh.T, 300)]
    pts += [0.5 * (mesh.xyz[a] + mesh.xyz[b]) for a, b, *_ in tn]  # edge midpoints
    pts += [(mesh.xyz[a] + mesh.xyz[b] + mesh.xyz[c]) / 3.0 for a, b, c, _ in tn]  # face centres
    hits = 0
    for p in pts:
        t_scan = orc.locate(mesh, p, hint=-1)
        assert fast.locate(mesh, p, hint=-1) == t_scan
        hits += t_scan >= 0
    assert 0.5 * len(pts) < hits < len(pts)
    sp = O.plasma_species(1e10, 1.0, 1.0, 0.05, 4)
    parts = O.seed_particles(mesh, sp, 4, 3)
    E = np.tile([4e4, -2e4, 1e4], (mesh.N, 1))  # strong field: multi-tet crossings
    for nb in (True, False):
        a = orc.push(mesh, E, parts, sp, 5e-8, neighbors=nb)
        b = fast.push(mesh, E, parts, sp, 5e-8, neighbors=nb)
        for k in ("x", "v", "tet", "lost", "rho"):
            assert np.array_equal(a[k], b[k]), k
        assert a["substeps"] == b["substeps"]
    fast.close()


def test_config0_push_matches_reference_fixture():
    """The oracle at the first benchmark configuration's full size (32^3 cells x 6 tets,
    1.29 M seeded particles) against the reference's push of a subsample (config0_ref.npz)."""
    from golden.make_golden import CONFIG0_STRIDE, config0_laplace, make_config0_inputs, subsample

    g = np.load(os.path.join(GOLDEN, "config0_ref.npz"))
    o = O.Oracle(fast_locate=True)
    mesh, sp, parts, dt = make_config0_inputs()
    A, phi = config0_laplace(o, mesh)
    assert np.sum(phi) == g["phi_sum"]
    E = o.lsq(mesh, A, phi, reg=1e-18)
    assert abs(np.sum(np.abs(E)) - g["E_abs_sum"]) <= 1e-12 * g["E_abs_sum"]
    out = o.push(mesh, E, subsample(parts, CONFIG0_STRIDE), sp, dt)
    assert np.array_equal(out["tet"], g["push_tet"]) and np.array_equal(out["lost"], g["push_lost"])
    assert out["substeps"] == int(g["push_substeps"])
    assert np.abs(out["x"] - g["push_x"]).max() < 1e-12 * np.abs(g["push_x"]).max()
    assert rel_err(out["v"], g["push_v"]) < 1e-12
    rho = np.zeros(mesh.N)
    rho[g["rho_nodes"]] = g["rho_vals"]
    assert rel_err(out["rho"], rho) < 1e-12
    o.close()
