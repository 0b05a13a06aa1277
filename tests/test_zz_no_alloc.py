"""The allocation-free CSR Jacobi-PCG entry point.

Some callers of this library cannot call cudaMalloc -- an application that owns a fixed
device-memory arena and passes only pointers into it, or code running where the allocator
is unavailable.  scdat_pcg_csr_noalloc serves them from a static device scratch array; this
test checks, through the C ABI, that two calls in a row give the result of the allocating
scdat_pcg_csr on the same system, and that an oversized system is refused.  The file is
named to be collected last.
"""
import os

import numpy as np
import pytest

from conftest import rel_err
from golden.make_golden import make_inputs
from pic_helpers import pcg_csr_on_device, reduced_system

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_noalloc_matches_allocating_entry_point(lib, orc):
    g = np.load(os.path.join(GOLDEN, "box6_body.npz"))
    mesh, *_ = make_inputs("box6_body")
    A = orc.assemble(mesh)
    rp, col, val, diag, b, inner = reduced_system(mesh, A, g["push_rho"], mesh.phi_bc)
    x0 = np.zeros_like(b)
    rc, x_ref, it_ref, rel_ref = pcg_csr_on_device(lib.scdat_pcg_csr, rp, col, val, diag, b, x0, 1e-14, 20000)
    assert rc == 0
    for _ in range(2):  # the scratch keeps the previous call's contents
        rc, x, it, rel = pcg_csr_on_device(lib.scdat_pcg_csr_noalloc, rp, col, val, diag, b, x0, 1e-14, 20000)
        assert rc == 0
        assert it == it_ref
        assert rel_err(x, x_ref) < 1e-12
        assert rel_err(x, g["phi_charge"][inner]) < 1e-12


def test_noalloc_rejects_oversized_system(lib):
    import ctypes as C

    it, rel = C.c_int32(), C.c_double()
    assert lib.scdat_pcg_csr_noalloc((1 << 18) + 1, None, None, None, None, None, None, 1e-8, 10, None,
                                     C.byref(it), C.byref(rel)) == -4
