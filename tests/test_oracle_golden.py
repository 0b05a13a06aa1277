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
