"""Host-side checks of the C ABI that need no GPU: the library loads, exports every entry
point declared in include/*.h, and its mesh builder equals the oracle's."""
import glob
import os
import re

import numpy as np

import oracle as O
from scdat_b200 import build, capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        names.update(re.findall(r"SCDAT_API\s+[\w\s\*]+?\b(scdat_\w+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol():
    build.build()
    L = capi.load()
    names = declared_symbols()
    assert len(names) >= 20
    for n in sorted(names):
        assert hasattr(L, n), n
    assert set(capi.EXPORTS) <= names
    assert L.scdat_version().startswith(b"scdat_b200")


def test_default_params():
    L = capi.load()
    p = capi.Params()
    L.scdat_default_params(p)
    assert p.deposit_kernel == capi.DEP_LINEAR and p.deposit_segments == 10
    assert p.adaptive_floor_ratio == 0.001 and p.poisson_charge_sign == -1 and p.use_neighbor_lists == 1


def test_kuhn_box_matches_oracle():
    for n, body in [((6, 5, 4), ((1, 3), (2, 4), (1, 2))), ((3, 3, 3), None)]:
        m = capi.kuhn_box_mesh(n, 0.05, body=body, bias=-7.0, wall=1.0)
        om = O.kuhn_box(n, 0.05, body=body, bias=-7.0, wall=1.0)
        assert np.array_equal(m["xyz"], om.xyz)
        assert np.array_equal(m["tet"], om.tet)
        assert np.array_equal(m["dirichlet"], om.dirichlet)
        assert np.array_equal(m["phi"], om.phi_bc)
        assert np.array_equal(m["hex_ijk"], om.hex_ijk)


def test_null_arguments_rejected():
    L = capi.load()
    assert L.scdat_create(None, None, None) == -1
    assert L.scdat_step(None, 1) == -1
    assert L.scdat_kuhn_box_mesh(0, 1, 1, 0.1, None, None, 0.0, 0.0, None, None, None, None, None, None, None,
                                 None) == -1
