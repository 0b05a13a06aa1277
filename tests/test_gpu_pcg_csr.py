"""The context-free CSR Jacobi-PCG entry point against the reference's Poisson solutions."""
import os

import numpy as np
import pytest

from conftest import rel_err
from golden.make_golden import make_inputs
from pic_helpers import pcg_csr_on_device, reduced_system

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("case", ["box6_body", "box5_open"])
def test_pcg_csr_matches_reference(lib, orc, case):
    g = np.load(os.path.join(GOLDEN, f"{case}.npz"))
    mesh, *_ = make_inputs(case)
    A = orc.assemble(mesh)
    rp, col, val, diag, b, inner = reduced_system(mesh, A, g["push_rho"], mesh.phi_bc)
    rc, x, it, rel = pcg_csr_on_device(lib.scdat_pcg_csr, rp, col, val, diag, b, np.zeros_like(b), 1e-15, 20000)
    assert rc in (0, -5) and rel < 1e-13
    assert rel_err(x, g["phi_charge"][inner]) < 1e-12


def test_pcg_csr_edge_cases(lib):
    # empty system is a no-op; a bad size is rejected
    import ctypes as C

    it, rel = C.c_int32(), C.c_double()
    assert lib.scdat_pcg_csr(0, None, None, None, None, None, None, 1e-8, 10, None, C.byref(it), C.byref(rel)) == 0
    assert lib.scdat_pcg_csr(-1, None, None, None, None, None, None, 1e-8, 10, None, C.byref(it), C.byref(rel)) == -1


# Systems on which Jacobi-PCG cannot converge, with the outcome a CPU run of the same
# iteration gives: a zero diagonal entry (infinite Jacobi weight: the residual turns
# non-finite) and an indefinite matrix whose first direction has p.Ap < 0 (CG breaks down at
# once, the residual stays at |b|).  Both must report NOT_CONVERGED, not success.
BREAKDOWN = {
    "zero_diagonal": (np.array([0, 1, 3, 4], np.int32), np.array([1, 0, 2, 1], np.int32),
                      np.array([-1.0, -1.0, -1.0, -1.0]), np.array([2.0, 0.0, 2.0]), np.array([1.0, 1.0, 1.0])),
    "indefinite": (np.array([0, 1, 2], np.int32), np.array([1, 0], np.int32), np.array([2.0, 2.0]),
                   np.array([1.0, 1.0]), np.array([1.0, -1.0])),
}


def _cpu_jacobi_pcg_breaks_down(rp, col, val, diag, b):
    A = np.diag(diag.astype(float))
    for r in range(len(diag)):
        for e in range(rp[r], rp[r + 1]):
            A[r, col[e]] = val[e]
    with np.errstate(all="ignore"):
        z = b / diag
        pAp = z @ (A @ z)
    return not (pAp > 0.0) or not np.all(np.isfinite(z))


@pytest.mark.parametrize("name", sorted(BREAKDOWN))
@pytest.mark.parametrize("entry", ["scdat_pcg_csr", "scdat_pcg_csr_noalloc"])
def test_pcg_csr_breakdown_is_not_converged(lib, name, entry):
    rp, col, val, diag, b = BREAKDOWN[name]
    assert _cpu_jacobi_pcg_breaks_down(rp, col, val, diag, b)
    rc, x, it, rel = pcg_csr_on_device(getattr(lib, entry), rp, col, val, diag, b, np.zeros_like(b), 1e-10, 100)
    assert rc == -5, (rc, it, rel)
    assert it < 100  # stopped by the breakdown, not by the cap
    assert not (rel <= 1e-10)


def test_mixed_refinement_pass_cap_reports_not_converged(lib, orc):
    """The mixed form's FP64 refinement stops after its pass cap; a tolerance below FP64
    rounding (1e-18) cannot be met, so the solve must report NOT_CONVERGED with the residual of
    the returned solution, long before the iteration cap."""
    from golden.make_golden import make_inputs
    from pic_helpers import gpu_domain

    mesh, sp, *_ = make_inputs("box6_body")
    dom = gpu_domain(mesh, 2e-8, precision=1, pcg_rtol=1e-18, pcg_max_iter=100000)
    dom.set_species(sp)
    dom.set_potential(mesh.phi_bc)
    assert dom.solve_field(allow_not_converged=True) == -5
    st = dom.stats()
    assert st["last_pcg_iterations"] < 100000
    assert 1e-18 < st["last_pcg_relres"] < 1e-12  # FP64 rounding level, above the target
    dom.close()
    # the same mesh at a reachable tolerance converges
    dom = gpu_domain(mesh, 2e-8, precision=1, pcg_rtol=1e-10, pcg_max_iter=100000)
    dom.set_species(sp)
    dom.set_potential(mesh.phi_bc)
    assert dom.solve_field() == 0 and dom.stats()["last_pcg_relres"] <= 1e-10
    dom.close()
