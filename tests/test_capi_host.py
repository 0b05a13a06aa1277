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


def test_create_failure_reason_outlives_the_context():
    """scdat_create frees a context it could not finish; scdat_last_error(NULL) still gives the
    calling thread's reason.  The mesh and parameter checks run on the host before any CUDA
    call, so this needs no GPU."""
    import ctypes as C

    L = capi.load()
    m = capi.kuhn_box_mesh((2, 2, 2), 0.1)
    xyz = np.ascontiguousarray(m["xyz"])
    tet = np.ascontiguousarray(m["tet"]).copy()
    dirichlet = np.ascontiguousarray(m["dirichlet"])
    p = capi.Params()
    L.scdat_default_params(p)
    p.dt = 1e-9
    md = capi.MeshDesc(len(xyz), len(tet), xyz.ctypes.data, tet.ctypes.data, None, dirichlet.ctypes.data, None)
    h = C.c_void_p()

    tet[3, 2] = len(xyz) + 5  # a node index past the end
    assert L.scdat_create(C.byref(md), C.byref(p), C.byref(h)) == -1
    assert not h.value
    assert L.scdat_last_error(None) == b"tet node index out of range"

    tet[3, 2] = 0
    p.dt = 0.0
    assert L.scdat_create(C.byref(md), C.byref(p), C.byref(h)) == -1
    assert L.scdat_last_error(None) == b"dt must be positive"

    md.n_nodes = 0
    assert L.scdat_create(C.byref(md), C.byref(p), C.byref(h)) == -1
    assert L.scdat_last_error(None) == b"empty mesh"

    assert L.scdat_create(None, None, None) == -1
    assert L.scdat_last_error(None) == b"scdat_create: null argument"
    # the Python wrapper reports the same reason
    bad = dict(m, tet=tet.copy())
    bad["tet"][0, 0] = -1
    try:
        capi.Domain(bad["xyz"], bad["tet"], bad["dirichlet"], 1e-9)
    except capi.ScdatError as e:
        assert "tet node index out of range" in str(e)
    else:
        raise AssertionError("a mesh with a negative node index was accepted")
