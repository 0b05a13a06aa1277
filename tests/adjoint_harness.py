"""Thin test harness: the device adjoint window (scdat_adjoint_window) as a
torch.autograd.Function of (bias, Te, delta_max), and its central finite-difference check with
frozen random streams (the particles are re-seeded with the same Philox draws, so a change of
Te only rescales their velocities)."""
import numpy as np
import torch

import oracle as O
from pic_helpers import gpu_domain, gpu_load_particles


class Window:
    """A small FP64 scenario: Kuhn box, a body with a floating dielectric surface circuit and
    Sternglass secondaries, electrons and H+; J = wV . mean face potential + wI . net current
    collected by the body over the window."""

    def __init__(self, n=(6, 6, 6), h=0.05, body=((2, 4), (2, 4), (2, 4)), density=3e10, ti=1.0, ppc=4, seed=33,
                 dt=2e-8, steps=8, checkpoint=3, e_max=300.0, wV=1.0, wI=0.0):
        self.n, self.h, self.body, self.density, self.ti, self.ppc, self.seed = n, h, body, density, ti, ppc, seed
        self.dt, self.steps, self.checkpoint, self.e_max = dt, steps, checkpoint, e_max
        self.blo = tuple(body[a][0] * h for a in range(3))
        self.bhi = tuple(body[a][1] * h for a in range(3))
        self.wV, self.wI = wV, wI

    def run(self, bias, te, dmax):
        mesh = O.kuhn_box(self.n, self.h, body=self.body, bias=bias)
        sp = O.plasma_species(self.density, te, self.ti, self.h, self.ppc)
        parts = O.seed_particles(mesh, sp, self.ppc, self.seed)
        dom = gpu_domain(mesh, self.dt, face_bc=(1,) * 6, pcg_rtol=1e-14, pcg_max_iter=20000)
        try:
            gpu_load_particles(dom, sp, parts)
            dom.set_surface_circuit(self.blo, self.bhi, eps_r=3.0, thickness=1e-3, v0=bias)
            dom.set_secondary_emission(1, dmax, self.e_max)
            dom.set_potential(mesh.phi_bc)
            dom.solve_field()
            gI = self.wI / (self.steps * self.dt)
            return dom.adjoint_window(self.steps, self.checkpoint, g_V=[self.wV / 6.0] * 6, g_Q=[gI] * 6, te_ev=te)
        finally:
            dom.close()


class WindowJ(torch.autograd.Function):
    """J(bias, Te, delta_max) with the device adjoint as its backward."""

    @staticmethod
    def forward(ctx, params, window):
        bias, te, dmax = (float(v) for v in params.detach().cpu())
        r = window.run(bias, te, dmax)
        ctx.save_for_backward(torch.tensor([r["dbias"], r["dte"], r["ddelta"]], dtype=torch.float64))
        return torch.tensor(r["J"], dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad):
        (g,) = ctx.saved_tensors
        return grad * g, None


def central_difference(window, params, rel=1e-4):
    """(J(p + h e_k) - J(p - h e_k)) / 2h per parameter, h = rel * |p_k|."""
    out = []
    for k in range(len(params)):
        h = rel * abs(params[k])
        up, dn = list(params), list(params)
        up[k] += h
        dn[k] -= h
        out.append((window.run(*up)["J"] - window.run(*dn)["J"]) / (2 * h))
    return np.array(out)


class BoxWindow:
    """The differentiation configuration at its size: a Kuhn box of n^3 cells (0.05 m) with a
    central body of n/4 cells per edge carrying the floating dielectric circuit, electrons and
    H+ at 1e10 m^-3 seeded on the device (the same Philox draws for every parameter set, so a
    change of Te rescales the electron velocities), Sternglass secondaries (Emax 300 eV);
    J = wV . mean face potential + wI . net current collected by the body over the window."""

    def __init__(self, n=48, ppc=32, steps=50, checkpoint=10, wV=1.0, wI=0.0, seed=4321):
        from scdat_b200 import capi

        self.n, self.ppc, self.steps, self.checkpoint, self.wV, self.wI, self.seed = n, ppc, steps, checkpoint, wV, wI, seed
        self.h, self.dt, self.density, self.ti, self.e_max = 0.05, 2e-8, 1e10, 1.0, 300.0
        q = n // 4
        lo = (n - q) // 2
        self.body = ((lo, lo + q),) * 3
        self.blo = tuple(b[0] * self.h for b in self.body)
        self.bhi = tuple(b[1] * self.h for b in self.body)
        self.mesh = capi.kuhn_box_mesh((n, n, n), self.h, body=self.body, bias=-1.0)

    def run(self, bias, te, dmax):
        from scdat_b200 import capi

        m = self.mesh
        phi = np.where(m["phi"] != 0.0, bias, 0.0)
        dom = capi.Domain(m["xyz"], m["tet"], m["dirichlet"], self.dt, face_bc=(1,) * 6, pcg_rtol=1e-14,
                          pcg_max_iter=20000)
        try:
            dom.set_species(O.plasma_species(self.density, te, self.ti, self.h, self.ppc))
            dom.seed_box(0, (self.n,) * 3, self.h, self.body, self.ppc, te, self.seed)
            dom.seed_box(1, (self.n,) * 3, self.h, self.body, self.ppc, self.ti, self.seed)
            dom.set_surface_circuit(self.blo, self.bhi, eps_r=3.0, thickness=1e-3, v0=bias)
            dom.set_secondary_emission(1, dmax, self.e_max)
            dom.set_potential(phi)
            dom.solve_field(allow_not_converged=True)
            gI = self.wI / (self.steps * self.dt)
            r = dom.adjoint_window(self.steps, self.checkpoint, g_V=[self.wV / 6.0] * 6, g_Q=[gI] * 6, te_ev=te)
            r["collected"] = int(np.asarray(dom.surface_state()["counts"]).sum())
            return r
        finally:
            dom.close()
