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
