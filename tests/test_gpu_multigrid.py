"""The lattice-multigrid preconditioner of the field solve (scdat_set_field_preconditioner).

The preconditioner changes how many CG iterations a solve takes, not what it converges to: at a
tight tolerance the multigrid-preconditioned solve gives the Jacobi-preconditioned solve's
potential (and the oracle's) to 1e-11, in both forms, alone and inside full PIC steps, in far
fewer iterations.  A mesh whose nodes are not on a lattice is refused."""
import numpy as np
import pytest

import oracle as O
from conftest import rel_err
from pic_helpers import gpu_domain, gpu_load_particles, gpu_state

pytestmark = pytest.mark.gpu


def _box(n):
    q = n // 4
    lo = (n - q) // 2
    return O.kuhn_box((n, n, n), 0.05, body=((lo, lo + q),) * 3, bias=-10.0)


def _charge(mesh, seed=3):
    rng = np.random.default_rng(seed)
    return rng.normal(0.0, 1e-13, mesh.N) * (mesh.dirichlet == 0)


def _solve(mesh, precision, precond, rtol, rho):
    from scdat_b200 import capi

    dom = gpu_domain(mesh, 2e-8, precision=precision, pcg_rtol=rtol, pcg_max_iter=20000)
    dom.set_species(O.plasma_species(1e10, 1.0, 1.0, 0.05, 2))
    if precond:
        dom.set_preconditioner(capi.PRECOND_MULTIGRID)
    dom.set_potential(mesh.phi_bc)
    dom.set_charge_density(rho)
    rc = dom.solve_field(allow_not_converged=True)
    _, phi, E = dom.fields()
    st = dom.stats()
    levels = dom.solver_levels()
    dom.close()
    return rc, phi, E, st["last_pcg_iterations"], st["last_pcg_relres"], levels


@pytest.mark.parametrize("n", [16, 32])
@pytest.mark.parametrize("precision", [0, 1])
def test_multigrid_gives_the_jacobi_solution(lib, n, precision):
    mesh = _box(n)
    rho = _charge(mesh)
    rtol = 1e-13 if precision == 0 else 1e-12
    rc_j, phi_j, E_j, it_j, rel_j, _ = _solve(mesh, precision, False, rtol, rho)
    rc_m, phi_m, E_m, it_m, rel_m, levels = _solve(mesh, precision, True, rtol, rho)
    print(f"n={n} precision={precision}: Jacobi {it_j} it ({rel_j:.1e}), multigrid {it_m} it ({rel_m:.1e}), "
          f"levels {levels}")
    assert len(levels) >= 2 and levels[-1][0] <= 1024
    assert rc_m == 0 and rel_m <= rtol
    assert rel_err(phi_m, phi_j) < 1e-11
    assert rel_err(E_m, E_j) < 1e-9
    assert it_m <= 30 and 3 * it_m < it_j


def test_multigrid_config0_matches_oracle(lib):
    """The 32^3 benchmark mesh, FP64 form: multigrid-preconditioned solve to 1e-14 against the
    oracle's Jacobi-PCG to 1e-14 from the same charge."""
    mesh = O.kuhn_box((32, 32, 32), 0.05, body=((12, 20),) * 3, bias=-10.0)
    o = O.Oracle()
    A = o.assemble(mesh)
    rho = _charge(mesh, 9)
    ref_phi, _, _ = o.poisson(mesh, A, rho, mesh.phi_bc, rtol=1e-14)
    rc, phi, E, it, rel, _ = _solve(mesh, 0, True, 1e-14, rho)
    assert rel_err(phi, ref_phi) < 1e-12
    assert rel_err(E, o.lsq(mesh, A, ref_phi)) < 1e-11
    assert it <= 30


@pytest.mark.parametrize("precision", [0, 1])
def test_multigrid_pic_steps_match_jacobi(lib, precision):
    """Four PIC steps with the field solved each step: the multigrid run reproduces the Jacobi
    run (FP64 form to 1e-12 at a 1e-14 solve; precision form within its FP32 push's rounding)."""
    from scdat_b200 import capi

    mesh = _box(16)
    sp = O.plasma_species(1e10, 1.0, 1.0, 0.05, 4)
    parts = O.seed_particles(mesh, sp, 4, 5)
    out = []
    for precond in (False, True):
        dom = gpu_domain(mesh, 2e-8, face_bc=(1,) * 6, precision=precision,
                         pcg_rtol=1e-14 if precision == 0 else 1e-11, pcg_max_iter=20000)
        gpu_load_particles(dom, sp, parts)
        if precond:
            dom.set_preconditioner(capi.PRECOND_MULTIGRID)
        dom.set_potential(mesh.phi_bc)
        dom.step(4)
        rho, phi, E = dom.fields()
        out.append((rho, phi, gpu_state(dom, len(sp), len(parts["tet"]))))
        dom.close()
    (r0, p0, s0), (r1, p1, s1) = out
    tol = 1e-12 if precision == 0 else 1e-6
    assert rel_err(p1, p0) < tol
    act = (s0["status"] == O.ACTIVE) & (s1["status"] == O.ACTIVE)
    assert (s0["status"] != s1["status"]).mean() < (1e-9 if precision == 0 else 1e-3)
    assert np.abs(s1["x"][act] - s0["x"][act]).max() < (1e-12 if precision == 0 else 1e-6)


def test_multigrid_refuses_a_non_lattice_mesh(lib):
    from scdat_b200 import capi

    mesh = _box(8)
    inner = np.nonzero(mesh.dirichlet == 0)[0]
    mesh.xyz[inner[len(inner) // 2]] += 0.003  # one node off the lattice
    dom = gpu_domain(mesh, 2e-8)
    with pytest.raises(capi.ScdatError) as e:
        dom.set_preconditioner(capi.PRECOND_MULTIGRID)
    assert e.value.rc == -1 and "lattice" in str(e.value)
    with pytest.raises(capi.ScdatError):
        dom.set_preconditioner(7)
    dom.set_preconditioner(capi.PRECOND_JACOBI)
    dom.close()
