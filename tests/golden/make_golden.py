"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run in a checkout where the reference tree is present and oracle/_ref was built
(`make -C oracle ref`):

    python tests/golden/make_golden.py            # the small cases
    python tests/golden/make_golden.py config0    # config0_ref.npz, the 32^3 configuration
    python tests/golden/make_golden.py sampler    # sampler_ref.npz, the surface current sampler

Every fixture is produced by the reference's own classes (CrossTetrahedron, PoissonSolver,
PICCycle, PicMccSurfaceCurrentSampler) through oracle/ref_harness.cpp on identical, seeded mesh
and particle state (the sampler seeds its own particles; its fixture holds its mesh and output).
The inputs are regenerated from the recorded seeds by oracle.py's builders.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

CASES = {
    # name: (n, h, body, bias, ppc, seed, dt, nsteps, face_bc)
    "box6_body": ((6, 6, 6), 0.05, ((2, 4), (2, 4), (2, 4)), -10.0, 4, 1234, 2e-8, 3, (2, 2, 2, 2, 1, 1)),
    "box5_open": ((5, 4, 6), 0.05, None, 0.0, 3, 77, 2e-8, 3, (1, 1, 1, 1, 1, 1)),
    "box4_strong": ((4, 4, 4), 0.05, ((1, 3), (1, 3), (1, 3)), -1000.0, 3, 9, 5e-8, 2, (2, 2, 2, 2, 1, 1)),
}


def make_inputs(case):
    n, h, body, bias, ppc, seed, dt, nsteps, face_bc = CASES[case]
    mesh = O.kuhn_box(n, h, body=body, bias=bias)
    sp = O.plasma_species(1e10, 1.0, 1.0, h, ppc)
    parts = O.seed_particles(mesh, sp, ppc, seed)
    return mesh, sp, parts, dt, nsteps, face_bc


# The first benchmark configuration at its full size: 32^3 hex cells of 0.05 m x 6 tets, the
# 8^3-cell body (cells 12..19 per axis) at -10 V, outer faces at 0 V, electrons and H+ at
# 1e10 m^-3 and 1 eV, 20 particles per cell per species, dt = 2e-8 s.
CONFIG0 = dict(n=(32, 32, 32), h=0.05, body=((12, 20), (12, 20), (12, 20)), bias=-10.0, ppc=20, seed=2024, dt=2e-8)
# every CONFIG0_STRIDE-th particle of the seeded population goes through the reference push
CONFIG0_STRIDE = 315


def make_config0_inputs():
    c = CONFIG0
    mesh = O.kuhn_box(c["n"], c["h"], body=c["body"], bias=c["bias"])
    sp = O.plasma_species(1e10, 1.0, 1.0, c["h"], c["ppc"])
    parts = O.seed_particles(mesh, sp, c["ppc"], c["seed"])
    return mesh, sp, parts, c["dt"]


def config0_laplace(o, mesh):
    """Laplace potential of the configuration by the oracle's CG to 1e-14 (the reference's dense
    PoissonSolver needs ~10 GB at this size); deterministic, so the GPU tests recompute it."""
    A = o.assemble(mesh)
    phi, _, _ = o.poisson(mesh, A, np.zeros(mesh.N), mesh.phi_bc, rtol=1e-14)
    return A, phi


def subsample(parts, stride):
    return {k: (v[::stride].copy() if isinstance(v, np.ndarray) and v.shape[:1] == parts["tet"].shape else v)
            for k, v in parts.items()}


def make_config0(o, r):
    mesh, sp, parts, dt = make_config0_inputs()
    _, phi = config0_laplace(o, mesh)
    E = r.lsq(mesh, phi)  # PICCycle::setPotential's LSQ field, by the reference
    sub = subsample(parts, CONFIG0_STRIDE)
    push = r.push(mesh, E, sub, sp, dt)  # CrossTetrahedron with neighbour lists filled
    nz = np.nonzero(push["rho"])[0]
    np.savez_compressed(
        os.path.join(HERE, "config0_ref.npz"),
        phi_sum=np.sum(phi), phi_abs_sum=np.sum(np.abs(phi)), E_abs_sum=np.sum(np.abs(E)),
        push_x=push["x"], push_v=push["v"], push_tet=push["tet"], push_lost=push["lost"],
        push_substeps=push["substeps"], rho_nodes=nz.astype(np.int32), rho_vals=push["rho"][nz],
    )
    print("config0", mesh.N, mesh.T, parts["x"].shape[0], sub["x"].shape[0])


# PicMccSurfaceCurrentSampler scenario: a 1 cm^2 plate 1 mm below the plasma boundary, 8 layers,
# a low-density Ar plasma (Debye length well above the gap, so the field is the applied one),
# MCC off, the sampler's default window and seed.
SAMPLER = dict(area_m2=1e-4, aspect=1.0, gap_m=1e-3, z_layers=8, ppe=2000, window_steps=12, seed=20260408,
               ne=1e12, ni=1e12, te_ev=5.0, ti_ev=0.2, ion_amu=40.0, reference_v=0.0, probe_dv=0.5)
SAMPLER_POTENTIALS = (-2.0, 0.0)


def make_sampler(r):
    c = SAMPLER
    xyz, tet = r.sampler_mesh(c["area_m2"], c["aspect"], c["gap_m"], c["z_layers"])
    rows = []
    for v in SAMPLER_POTENTIALS:
        out = r.sampler_sample(c["area_m2"], c["gap_m"], c["z_layers"], c["ppe"], c["window_steps"], c["seed"],
                               c["ne"], c["ni"], c["te_ev"], c["ti_ev"], c["ion_amu"], v, c["reference_v"],
                               c["probe_dv"])
        assert out["valid"] == 1.0
        rows.append([out[k] for k in ("electron", "ion", "emitted", "net", "derivative", "segments")])
    np.savez_compressed(os.path.join(HERE, "sampler_ref.npz"), xyz=xyz, tet=tet,
                        potentials=np.array(SAMPLER_POTENTIALS), samples=np.array(rows))
    print("sampler", xyz.shape[0], tet.shape[0], np.array(rows))


def main():
    o = O.Oracle()
    r = O.Reference()
    if len(sys.argv) > 1 and sys.argv[1] == "config0":
        make_config0(O.Oracle(fast_locate=True), r)
        r.close()
        return
    if len(sys.argv) > 1 and sys.argv[1] == "sampler":
        make_sampler(r)
        r.close()
        return
    for case in CASES:
        mesh, sp, parts, dt, nsteps, face_bc = make_inputs(case)
        A = o.assemble(mesh)
        # Laplace field the reference solves (fresh PoissonSolver, DIRECT)
        phi_l, E_l = r.poisson(mesh, np.zeros(mesh.N), mesh.phi_bc)
        push = r.push(mesh, E_l, parts, sp, dt)
        # Poisson with the deposited charge
        phi_q, E_q = r.poisson(mesh, push["rho"], mesh.phi_bc)
        cyc = r.cycle(mesh, parts, sp, nsteps, dt, face_bc, phi_l)
        np.savez_compressed(
            os.path.join(HERE, f"{case}.npz"),
            phi_laplace=phi_l, E_laplace=E_l,
            push_x=push["x"], push_v=push["v"], push_tet=push["tet"], push_lost=push["lost"], push_rho=push["rho"],
            push_substeps=push["substeps"],
            phi_charge=phi_q, E_charge=E_q,
            cyc_x=cyc["x"], cyc_v=cyc["v"], cyc_id=cyc["id"], cyc_status=cyc["status"], cyc_rho=cyc["rho"],
            cyc_phi=cyc["phi"], cyc_E=cyc["E"], cyc_ledger=cyc["ledger"], cyc_stats=cyc["stats"],
        )
        print(case, mesh.N, mesh.T, parts["x"].shape[0])
    r.close()


if __name__ == "__main__":
    main()
