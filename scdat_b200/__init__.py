"""scdat_b200 -- B200-native PIC-MCC step and per-step Poisson solve for SCDAT.

The product is the CUDA library libscdat_b200.so behind the C ABI in include/scdat_b200.h
(built by ``python -m scdat_b200.build``) and the C++20 host classes in scdat_b200/host/
that mirror SCDAT's PICCycle / CrossTetrahedron / PoissonSolver interfaces.  The Python
module ``scdat_b200.capi`` is a ctypes binding of the same C ABI for tests and benchmarks.
"""
__version__ = "0.1.0"
