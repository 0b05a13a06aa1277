"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run in a checkout where the reference tree is present and oracle/_ref was built
(`make -C oracle ref`):

    python tests/golden/make_golden.py

Every fixture is produced by the reference's own classes (CrossTetrahedron, PoissonSolver,
PICCycle) through oracle/ref_harness.cpp on identical, seeded mesh and particle state.
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


def main():
    o = O.Oracle()
    r = O.Reference()
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
