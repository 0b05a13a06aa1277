"""The hand-written adjoint window against central finite differences (relative step 1e-4,
frozen Philox streams), through the torch.autograd.Function harness.

J is the mean face potential of a floating dielectric body (and, in the second case, the net
current it collects, secondaries included) after an 8-step FP64 window checkpointed every 3
steps; the parameters are the body bias, the electron temperature and the Sternglass peak."""
import numpy as np
import pytest
import torch

from adjoint_harness import Window, WindowJ, central_difference

pytestmark = pytest.mark.gpu
P0 = [-8.0, 2.0, 2.0]  # bias [V], Te [eV], delta_max


@pytest.mark.parametrize("wV,wI", [(1.0, 0.0), (1.0, 1e3)])
def test_adjoint_matches_central_differences(lib, wV, wI):
    w = Window(wV=wV, wI=wI)
    p = torch.tensor(P0, dtype=torch.float64, requires_grad=True)
    J = WindowJ.apply(p, w)
    J.backward()
    adj = p.grad.numpy()
    fd = central_difference(w, P0)
    print("adjoint", adj, "fd", fd)
    assert np.all(np.isfinite(adj)) and abs(adj[0]) > 0 and abs(adj[1]) > 0 and abs(adj[2]) > 0
    np.testing.assert_allclose(adj, fd, rtol=1e-3, atol=1e-3 * np.abs(fd).max())


def test_adjoint_window_leaves_the_run_at_its_end(lib):
    """The window advances the context like scdat_step: the same final state."""
    import oracle as O
    from pic_helpers import gpu_domain, gpu_load_particles, gpu_state

    w = Window()
    out = []
    for use_adjoint in (True, False):
        mesh = O.kuhn_box(w.n, w.h, body=w.body, bias=P0[0])
        sp = O.plasma_species(w.density, P0[1], w.ti, w.h, w.ppc)
        parts = O.seed_particles(mesh, sp, w.ppc, w.seed)
        dom = gpu_domain(mesh, w.dt, face_bc=(1,) * 6, pcg_rtol=1e-14, pcg_max_iter=20000)
        gpu_load_particles(dom, sp, parts)
        dom.set_surface_circuit(w.blo, w.bhi, eps_r=3.0, thickness=1e-3, v0=P0[0])
        dom.set_secondary_emission(1, P0[2], w.e_max)
        dom.set_potential(mesh.phi_bc)
        dom.solve_field()
        if use_adjoint:
            dom.adjoint_window(w.steps, w.checkpoint, g_V=[1 / 6.0] * 6)
        else:
            dom.step(w.steps)
        out.append((dom.fields()[1], dom.surface_state()["V"], gpu_state(dom, len(sp), len(parts["tet"]))))
        dom.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2]["x"], out[1][2]["x"], equal_nan=True)


def test_adjoint_at_the_differentiation_configuration(lib):
    """48^3 cells x 6 tets, 32 ppc per species (7 M particles), Sternglass secondaries
    (delta_max 2, Emax 300 eV), a 50-step window checkpointed every 10: the adjoint gradients of
    the body potential and of the collected current in bias, Te and delta_max against central
    differences with frozen streams, to 1e-3.  The difference step is 1e-5 relative: at 1e-4 the
    +h and -h runs of this size already collect a different number of macro-particles, a
    discrete event whose charge jump the pathwise derivative holds fixed by construction, so
    the check first asserts that the two runs took the same collection choices."""
    from adjoint_harness import BoxWindow

    p0 = [-8.0, 1.0, 2.0]
    for wV, wI in ((1.0, 0.0), (0.0, 1e3)):
        w = BoxWindow(wV=wV, wI=wI)
        r = w.run(*p0)
        assert r["flags"] == 0  # no particle overflowed the sub-step replay tape
        adj = np.array([r["dbias"], r["dte"], r["ddelta"]])
        fd = []
        for k in range(3):
            hk = 1e-5 * abs(p0[k])
            up, dn = list(p0), list(p0)
            up[k] += hk
            dn[k] -= hk
            ru, rd = w.run(*up), w.run(*dn)
            assert ru["collected"] == rd["collected"] == r["collected"]
            fd.append((ru["J"] - rd["J"]) / (2 * hk))
        fd = np.array(fd)
        print("J weights", wV, wI, "adjoint", adj, "fd", fd)
        assert np.all(np.abs(adj - fd) <= 1e-3 * np.abs(fd))
