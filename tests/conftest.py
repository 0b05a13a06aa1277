"""Test configuration: the `gpu` marker, shared fixtures and the parity helpers.

`-m "not gpu"` runs the oracle, its pin against the reference, the golden fixtures and the
host-side checks on CPU.  `-m gpu` runs the CUDA library through its C ABI against the
oracle (and, where oracle/_ref was built, against the reference itself).
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def orc():
    import oracle

    return oracle.Oracle()


@pytest.fixture(scope="session")
def ref():
    import oracle

    if not oracle.reference_available():
        pytest.skip("reference library oracle/_ref/libscdat_ref.so not built")
    r = oracle.Reference()
    yield r
    r.close()


def gpu_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def lib():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from scdat_b200 import build, capi

    build.build()
    return capi.load()


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)
