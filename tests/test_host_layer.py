"""The C++20 host layer (scdat_b200/host): the reference's PIC-path classes over the C ABI.

CPU: the re-hosted reference tests (tests/cpp/test_host_layer.cpp) compile and link against
libscdat_host.so.  GPU: they pass, and a cycle driven through PICCycle / ParticleManager
matches the oracle's cycle on the same particles to 1e-12 relative."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import ROOT, rel_err
from pic_helpers import oracle_cycle

PKG = os.path.join(ROOT, "scdat_b200")
SRC = os.path.join(ROOT, "tests", "cpp", "test_host_layer.cpp")
EXE = os.path.join(PKG, "_build", "test_host_layer")
TOL = 1e-12


def _build_exe():
    from scdat_b200 import build

    build.build()
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    deps = [SRC, build.HOST_LIB, os.path.join(build.HOST_DIR, "scdat_host.hpp")]
    if os.path.exists(EXE) and os.path.getmtime(EXE) >= max(os.path.getmtime(d) for d in deps):
        return EXE
    cmd = ["g++", "-std=c++20", "-O1", "-Wall", SRC, f"-I{build.HOST_DIR}", f"-I{os.path.join(ROOT, 'include')}",
           f"-L{PKG}", "-lscdat_host", "-lscdat_b200", f"-Wl,-rpath,{PKG}", "-o", EXE]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return EXE


def test_host_layer_builds_and_links():
    exe = _build_exe()
    assert os.path.exists(exe)
    # every class of the mirrored interface is in the library
    r = subprocess.run(["nm", "-DC", os.path.join(PKG, "libscdat_host.so")], capture_output=True, text=True)
    for sym in ("SCDAT::PICcore::PICCycle::executeTimeStep()", "SCDAT::PICcore::PICCycle::initialize()",
                "SCDAT::FieldSolver::PoissonSolver::solve(", "SCDAT::Particle::ParticleManager::createElectron(",
                "SCDAT::Collision::executeBackgroundMccStep("):
        assert sym in r.stdout, sym


@pytest.mark.gpu
def test_reference_tests_pass_on_host_layer(lib):
    r = subprocess.run([_build_exe()], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("[  OK  ]") == 7


def _write_case(path, n, h, dt, nsteps, face_bc, phi0, kinds, x, v, w):
    with open(path, "wb") as f:
        np.array([*n, nsteps, *face_bc], np.int32).tofile(f)
        np.array([h, dt], np.float64).tofile(f)
        np.array([len(kinds)], np.int64).tofile(f)
        phi0.astype(np.float64).tofile(f)
        for k, xi, vi in zip(kinds, x, v):
            np.array([k], np.int32).tofile(f)
            np.concatenate([xi, vi, [w[k]]]).astype(np.float64).tofile(f)


@pytest.mark.gpu
def test_picycle_host_layer_matches_oracle(lib, orc, tmp_path):
    """PICCycle::executeTimeStep through the host layer, particles created by ParticleManager
    without location hints (first step locates them), against the oracle's cycle."""
    n, h, dt, nsteps = (4, 4, 4), 0.05, 2e-8, 3
    face_bc = (2, 2, 2, 2, 1, 1)
    mesh = O.kuhn_box(n, h, body=None, wall=0.0)
    # outer nodes: a potential ramp in z so the field is non-trivial
    phi0 = np.where(mesh.dirichlet == 1, -5.0 * mesh.xyz[:, 2] / (n[2] * h), 0.0)
    mesh.phi_bc = phi0.copy()
    w = 1e10 * h ** 3 / 4
    sp = [O.Species(-O.QE, O.ME, w, 0, 1.0), O.Species(O.QE, O.MP, w, 1, 1.0)]
    rng = np.random.default_rng(5)
    npart = 400
    kinds = np.repeat([0, 1], npart // 2).astype(np.int32)
    x = rng.uniform(0.01, n[0] * h - 0.01, size=(npart, 3))
    sig = np.where(kinds == 0, 4.19e5, 9.79e3)[:, None]
    v = rng.normal(size=(npart, 3)) * sig
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    _write_case(inp, n, h, dt, nsteps, face_bc, phi0, kinds, x, v, [w, w])
    r = subprocess.run([_build_exe(), "parity", str(inp), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    res = np.fromfile(out, np.float64)
    P = res[: 7 * npart].reshape(npart, 7)
    rho = res[7 * npart: 7 * npart + mesh.N]
    phi = res[7 * npart + mesh.N: 7 * npart + 2 * mesh.N]
    led = res[7 * npart + 2 * mesh.N: 7 * npart + 2 * mesh.N + 42].reshape(6, 7)
    sc = res[-1]

    parts = dict(x=x, v=v, tet=-np.ones(npart, np.int32), species=kinds, id=np.arange(npart))
    ref = oracle_cycle(orc, mesh, sp, parts, nsteps, dt, face_bc, phi0, rtol=1e-15)
    status = P[:, 6].astype(np.uint8)
    assert np.array_equal(status, ref["status"])
    act = status == O.ACTIVE
    assert act.sum() > npart // 2
    assert np.abs(P[act, :3] - ref["x"][act]).max() <= TOL * np.abs(ref["x"]).max()
    assert rel_err(P[act, 3:6], ref["v"][act]) < TOL
    assert rel_err(rho, ref["rho"]) < TOL
    assert rel_err(phi, ref["phi"]) < 1e-10
    assert np.array_equal(led[:, 4:6], ref["ledger"][:6, 4:6])
    np.testing.assert_allclose(led[:, [0, 1, 3]], ref["ledger"][:6, [0, 1, 3]], rtol=TOL, atol=1e-30)
    np.testing.assert_allclose(sc, ref["surface_charge"], rtol=TOL, atol=1e-30)


def test_collision_helpers_match_reference(ref, tmp_path):
    """The host layer's parseCollisionCrossSectionSetId and estimateCollisionBackgroundDensities
    against the reference's own (CollisionPicAdapter.cpp:212-282) on CPU: case folding and
    aliases of the set names; floors sanitised (non-finite or negative -> 0) and raised by the
    electron-like, ion-like and neutral weight densities of the active particles."""
    exe = _build_exe()
    for name in ("background_mcc_v1", "Background", "DEFAULT", "BackgroundMccV1", "surfacePIC", "surface_pic",
                 "Surface_Pic_V1", "ArcPic", "vacuumarcpicv1", "arcpic_background_v1", "VACUUM_ARC_PIC_V1", "nonsense",
                 "", "background_mcc_v2"):
        r = subprocess.run([exe, "parse", name], capture_output=True, text=True, timeout=30)
        assert r.returncode == 0
        assert int(r.stdout) == ref.parse_cross_section_set(name), name
    rng = np.random.default_rng(4)
    types = (1, 20, 52, 0)  # electron, proton, ion, unknown (classified by the sign of its charge)
    for trial in range(12):
        n = int(rng.integers(0, 60))
        t = rng.choice(types, n)
        q = np.where(rng.random(n) < 0.3, 0.0, rng.choice([-1.0, 1.0], n) * 1.602176634e-19)
        w = np.where(rng.random(n) < 0.1, -1.0, rng.uniform(0.0, 1e6, n))
        act = (rng.random(n) < 0.8).astype(np.uint8)
        vol = [1e-6, 0.0, -1.0, np.inf, 2.5e-3][trial % 5]
        floors = np.array([[1e14, 0.0, 3e12], [np.nan, -5.0, np.inf], [0.0, 1e9, 1e9]][trial % 3])
        case = tmp_path / f"case{trial}.bin"
        with open(case, "wb") as f:
            np.array([n], np.int64).tofile(f)
            np.stack([t.astype(float), q, w, act.astype(float)], axis=1).astype(np.float64).tofile(f)
            np.array([vol, *floors], np.float64).tofile(f)
        out = tmp_path / f"out{trial}.bin"
        r = subprocess.run([exe, "densities", str(case), str(out)], capture_output=True, text=True, timeout=30)
        assert r.returncode == 0, r.stdout + r.stderr
        mine = np.fromfile(out, np.float64)
        theirs = ref.estimate_densities(t, q, w, act, vol, floors)
        np.testing.assert_array_equal(mine, theirs)
