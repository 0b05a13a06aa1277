"""Batched scenarios (scdat_batch): several independent mixed-precision scenarios of different
sizes stepped together by one launch per kernel and one CUDA-graph launch per step.

A one-scenario batch gives every launch the same block partition as the single-context step,
so its results are bitwise those of scdat_step.  With several scenarios the field reductions
are partitioned differently: the first step's fixed-point charge is still bitwise, its
potential agrees to the solver tolerance, and later steps agree to the FP32 push's rounding
(1e-5, the error budget of the mixed form).  The graph and the host-driven loop are bitwise
equal."""
import numpy as np
import pytest

import oracle as O
from conftest import rel_err
from pic_helpers import gpu_domain, gpu_load_particles, gpu_state

pytestmark = pytest.mark.gpu

SCEN = [  # (cells, body, bias, density, Te, ppc, seed)
    ((6, 6, 6), ((2, 4), (2, 4), (2, 4)), -5.0, 1e10, 1.0, 4, 11),
    ((8, 5, 7), ((3, 5), (2, 3), (3, 4)), -20.0, 3e10, 2.0, 3, 12),
    ((5, 5, 5), None, 0.0, 1e9, 0.5, 5, 13),
]


def _scenario(k, mcc=True):
    cells, body, bias, n0, te, ppc, seed = SCEN[k]
    h = 0.05
    mesh = O.kuhn_box(cells, h, body=body, bias=bias)
    sp = O.plasma_species(n0, te, te, h, ppc)
    parts = O.seed_particles(mesh, sp, ppc, seed)
    dom = gpu_domain(mesh, 2e-8, face_bc=(2, 2, 2, 2, 1, 1), precision=1, pcg_rtol=1e-10, sort_interval=2)
    gpu_load_particles(dom, sp, parts)
    if mcc:
        for s in range(len(sp)):
            dom.set_elastic(s, 1e18, 1e-19)
    dom.set_potential(mesh.phi_bc)
    return dom, sp, parts


def _state(dom, sp, parts):
    rho, phi, E = dom.fields()
    return dict(rho=rho, phi=phi, E=E, ledger=dom.ledger(), **gpu_state(dom, len(sp), len(parts["tet"])))


def test_single_scenario_batch_is_bitwise_the_single_step(lib):
    from scdat_b200 import capi

    dom, sp, parts = _scenario(0)
    dom.step(3)
    ref = _state(dom, sp, parts)
    dom.close()
    dom, sp, parts = _scenario(0)
    b = capi.Batch([dom])
    b.step(3)
    got = _state(dom, sp, parts)
    steps = dom.stats()["completed_steps"]
    b.close()
    dom.close()
    for key in ("rho", "phi", "E", "ledger", "x", "v", "tet", "status"):
        assert np.array_equal(np.nan_to_num(got[key]), np.nan_to_num(ref[key])), key
    assert steps == 3


def test_batch_over_a_pending_resort_is_bitwise_the_single_step(lib):
    """A context whose last step re-sorted (the precision form leaves that re-sort's gather to
    the next push) joins a batch, which gathers the store first: two more steps in the batch
    give bitwise what four steps of the context alone give, where the third step's push read
    the store through the permutation."""
    from scdat_b200 import capi

    dom, sp, parts = _scenario(0)
    dom.step(4)
    ref = _state(dom, sp, parts)
    dom.close()
    dom, sp, parts = _scenario(0)
    dom.step(2)  # sort_interval 2: re-sorted after the second step
    b = capi.Batch([dom])
    b.step(2)
    got = _state(dom, sp, parts)
    b.close()
    dom.close()
    for key in ("rho", "phi", "E", "ledger", "x", "v", "tet", "status"):
        assert np.array_equal(np.nan_to_num(got[key]), np.nan_to_num(ref[key])), key


def test_batch_of_uneven_scenarios_matches_single_steps(lib):
    from scdat_b200 import capi

    refs = []
    for k in range(len(SCEN)):
        dom, sp, parts = _scenario(k)
        dom.step(1)
        first = dom.fields()[:2]
        dom.step(2)
        refs.append((first, _state(dom, sp, parts)))
        dom.close()
    doms = [_scenario(k) for k in range(len(SCEN))]
    b = capi.Batch([d for d, _, _ in doms])
    try:
        b.step(1)
        first = [dom.fields()[:2] for dom, _, _ in doms]
        b.step(2)
        got = [(_state(dom, sp, parts), dom.stats()) for dom, sp, parts in doms]
    finally:
        b.close()
        for d, _, _ in doms:
            d.close()
    for k in range(len(SCEN)):
        assert np.array_equal(first[k][0], refs[k][0][0]), "first-step charge is exact"
        assert rel_err(first[k][1], refs[k][0][1]) < 1e-8
        (g, st), ref = got[k], refs[k][1]
        assert rel_err(g["phi"], ref["phi"]) < 1e-5
        act = (g["status"] == O.ACTIVE) & (ref["status"] == O.ACTIVE)
        assert (g["status"] != ref["status"]).mean() < 0.01
        assert np.abs(g["x"][act] - ref["x"][act]).max() < 1e-5
        assert st["completed_steps"] == 3 and st["last_pcg_relres"] < 1e-9


def test_graph_and_host_loop_agree(lib):
    from scdat_b200 import capi

    out = []
    for use_graph in (True, False):
        doms = [_scenario(k) for k in range(len(SCEN))]
        b = capi.Batch([d for d, _, _ in doms], use_graph=use_graph)
        b.step(3)
        out.append([_state(d, sp, parts) for d, sp, parts in doms])
        b.close()
        for d, _, _ in doms:
            d.close()
    for g, e in zip(out[0], out[1]):
        for key in ("rho", "phi", "x", "status"):
            assert np.array_equal(np.nan_to_num(g[key]), np.nan_to_num(e[key])), key


def test_autotune_picks_a_valid_shape(lib):
    from scdat_b200 import capi

    doms = [_scenario(k, mcc=False) for k in range(len(SCEN))]
    b = capi.Batch([d for d, _, _ in doms])
    t = b.autotune(1)
    assert t["push_blocks_per_sm"] in (2, 4, 8) and t["field_blocks_per_sm"] in (4, 8)
    b.step(1)
    assert b.last_step_ms() > 0
    assert all(d.stats()["completed_steps"] == 7 for d, _, _ in doms)
    b.close()
    for d, _, _ in doms:
        d.close()


def test_batch_rejects_fp64_contexts(lib):
    from scdat_b200 import capi

    mesh = O.kuhn_box((3, 3, 3), 0.05)
    dom = gpu_domain(mesh, 2e-8, precision=0)
    dom.set_species(O.plasma_species(1e10, 1.0, 1.0, 0.05, 1))
    with pytest.raises(capi.ScdatError):
        capi.Batch([dom])
    dom.close()


def test_batch_lifetime(lib):
    """A batch's graph and job tables point into its contexts' buffers.  The library refuses to
    destroy a context while a batch holds it; Domain.close closes such a batch first (also when
    the garbage collector finalises both in either order); and a batch destroyed before its
    contexts leaves nothing behind: a new context afterwards steps bitwise as in a process that
    never had a batch."""
    from scdat_b200 import capi

    dom, sp, parts = _scenario(0)
    dom.step(2)
    ref = _state(dom, sp, parts)
    dom.close()

    dom, sp, parts = _scenario(1)
    b = capi.Batch([dom])
    b.step(2)
    assert lib.scdat_destroy(dom.h) == -3  # SCDAT_ERR_STATE: held by a batch
    assert b"batch" in lib.scdat_last_error(dom.h)
    dom.close()  # closes the batch, then the context
    assert b.h is None and dom.h is None

    dom, sp, parts = _scenario(1)
    b = capi.Batch([dom])
    b.step(1)
    b.close()  # batch first, then the context
    assert lib.scdat_destroy(dom.h) == 0
    dom.h = None

    dom, sp, parts = _scenario(0)
    dom.step(2)
    got = _state(dom, sp, parts)
    dom.close()
    for key in ("rho", "phi", "E", "ledger", "x", "v", "tet", "status"):
        assert np.array_equal(np.nan_to_num(got[key]), np.nan_to_num(ref[key])), key
