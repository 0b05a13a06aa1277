"""Shared drivers for the parity tests: the oracle's PIC cycle in the reference's order
(PICCycle::executeTimeStep, Tools/PICcore/src/PICCycle.cpp:311-416) and the same cycle on
the CUDA library through its C ABI."""
import numpy as np

import oracle as O


def oracle_cycle(o, mesh, sp, parts, nsteps, dt, face_bc, phi0, neighbors=True, rtol=1e-15, body_tally=False,
                 surface=None):
    """surface: an O.SurfaceCircuit advanced after every push (body_tally implied)."""
    A = o.assemble(mesh)
    E = o.lsq(mesh, A, phi0, reg=1e-18)
    L = mesh.xyz.max(axis=0) - mesh.xyz.min(axis=0)
    period = tuple(L[a] if (face_bc[2 * a] == 2 or face_bc[2 * a + 1] == 2) else 0.0 for a in range(3))
    st = dict(x=parts["x"].copy(), v=parts["v"].copy(), tet=parts["tet"].copy(),
              status=np.zeros(len(parts["tet"]), np.uint8))
    phi = phi0.copy()
    ledger = np.zeros((7, 8))
    sc = 0.0
    rho = np.zeros(mesh.N)
    substeps = 0
    phi_bc = mesh.phi_bc.copy()
    if surface is not None:
        body_tally = True
        phi_bc = surface.apply(phi_bc)
    lo, hi = mesh.xyz.min(axis=0), mesh.xyz.max(axis=0)
    otol = max(1e-10, 1e-8 * float(np.max(hi - lo)))
    for _ in range(nsteps):
        before = st["status"].copy()
        out = o.push(mesh, E, dict(parts, x=st["x"], v=st["v"], tet=st["tet"]), sp, dt, status=st["status"],
                     neighbors=neighbors)
        out = o.boundary(mesh, out, parts, sp, face_bc, period=period, neighbors=neighbors, body_tally=body_tally)
        ledger += out["ledger"]
        sc += out["surface_charge"]
        substeps += out["substeps"]
        st = dict(x=out["x"], v=out["v"], tet=out["tet"], status=out["status"])
        rho = out["rho"]
        if surface is not None:
            # particles that left the mesh this step inside the domain box went into the body
            x = out["x"]
            into = (before == O.ACTIVE) & (out["status"] == O.ESCAPED) & np.all((x >= lo - otol) & (x <= hi + otol),
                                                                                axis=1)
            spi = parts["species"][into]
            qw = np.array([sp[s].q * sp[s].w for s in spi])
            m = np.array([sp[s].m for s in spi])
            ke = 0.5 * m * np.sum(out["v"][into] ** 2, axis=1) if len(spi) else np.zeros(0)
            ele = np.array([1.0 if sp[s].kind == 0 else 0.0 for s in spi])
            dq, emitted = surface.collect(x[into], qw, ke / O.QE, ele)
            ledger[6, 2] += emitted
            surface.advance(dq, dt)
            phi_bc = surface.apply(phi_bc)
        phi, _, _ = o.poisson(mesh, A, rho, phi_bc, rtol=rtol, phi0=phi)
        E = o.lsq(mesh, A, phi)
    return dict(st, rho=rho, phi=phi, E=E, ledger=ledger, surface_charge=sc, substeps=substeps)


def oracle_mcc_run(o, mesh, sp, parts, nsteps, dt, face_bc, n_t, sigma, seed, rtol=1e-15, mode=0):
    """The oracle's PIC-MCC run in the reference's order: each step the cycle (push, boundary
    events, field), then elastic MCC on the Philox streams of (seed, particle id, step), then
    the absorbed particles leave the container (Collision::executeBackgroundMccStep,
    CollisionPicAdapter.cpp:338-434).  Mode 2 (null collision) takes each species' speed bound
    from the previous push, as the device does.  Returns the active particles, the summed
    ledger, the collisions and the last fields."""
    procs = [O.Elastic(n_t, sigma, 1.0, 0.0, 0.0, 1, 0) for _ in sp]
    cur = {k: v.copy() for k, v in parts.items()}
    phi, ledger, hits = mesh.phi_bc.copy(), np.zeros((7, 8)), 0
    out = None
    vmax = None
    for k in range(nsteps):
        out = oracle_cycle(o, mesh, sp, cur, 1, dt, face_bc, phi, rtol=rtol)
        ledger += out["ledger"]
        phi = out["phi"]
        v = out["v"]
        if n_t > 0:
            v, h = o.mcc(out["v"], cur["species"], out["status"], cur["id"], sp, procs, dt, seed, k, mode=mode,
                         vmax=vmax)
            hits += h
        vmax = O.push_speed_bound(out["v"], cur["species"], out["status"], len(sp))
        act = out["status"] == O.ACTIVE
        cur = {key: val[act] for key, val in cur.items()}
        cur.update(x=out["x"][act], v=v[act], tet=out["tet"][act])
    return dict(parts=cur, ledger=ledger, hits=hits, rho=out["rho"], phi=out["phi"], E=out["E"])


def species_split(parts, s):
    m = parts["species"] == s
    return {k: (v[m] if isinstance(v, np.ndarray) and v.shape[:1] == m.shape else v) for k, v in parts.items()}


def gpu_domain(mesh, dt, face_bc=(0,) * 6, precision=0, neighbors=True, **kw):
    from scdat_b200 import capi

    return capi.Domain(mesh.xyz, mesh.tet, mesh.dirichlet, dt, nbr=mesh.nbr, precision=precision, face_bc=face_bc,
                       use_neighbor_lists=neighbors, **kw)


def gpu_load_particles(dom, sp, parts):
    """Species-major upload; returns the index map (device order -> oracle particle index)."""
    dom.set_species(sp)
    order = []
    for s in range(len(sp)):
        idx = np.nonzero(parts["species"] == s)[0]
        dom.set_particles(s, parts["x"][idx], parts["v"][idx], parts["tet"][idx], parts["id"][idx].astype(np.uint32))
        order.append(idx)
    return order


def gpu_state(dom, nspecies, nparts):
    """Device particles scattered back into oracle particle order (by id)."""
    x = np.full((nparts, 3), np.nan)
    v = np.full((nparts, 3), np.nan)
    tet = np.full(nparts, -9, np.int32)
    status = np.full(nparts, 255, np.uint8)
    for s in range(nspecies):
        g = dom.get_particles(s)
        ids = g["id"].astype(np.int64)
        x[ids] = g["x"]
        v[ids] = g["v"]
        tet[ids] = g["tet"]
        status[ids] = g["status"]
    return dict(x=x, v=v, tet=tet, status=status)


def reduced_system(mesh, A, rho, phi_bc, charge_sign=-1.0):
    """The Dirichlet-eliminated system of the interior rows (LinearSystem.cpp:37-58) in CSR:
    (row_ptr, col, val, diag, b, interior node ids)."""
    inner = np.nonzero(mesh.dirichlet == 0)[0]
    row_of = -np.ones(mesh.N, np.int64)
    row_of[inner] = np.arange(len(inner))
    rp, cols, vals, b = [0], [], [], np.zeros(len(inner))
    for r, n in enumerate(inner):
        bi = charge_sign * rho[n] * A["cv"][n]
        for e in range(A["rowptr"][n], A["rowptr"][n + 1]):
            j = A["col"][e]
            if mesh.dirichlet[j]:
                bi -= A["offw"][e] * phi_bc[j]
            else:
                cols.append(row_of[j])
                vals.append(A["offw"][e])
        b[r] = bi
        rp.append(len(cols))
    return (np.array(rp, np.int32), np.array(cols, np.int32), np.array(vals, np.float64),
            A["diag"][inner].copy(), b, inner)


def pcg_csr_on_device(entry, rp, col, val, diag, b, x0, rtol, max_iter):
    """Call a scdat_pcg_csr-shaped entry point on device copies (torch owns the memory)."""
    import ctypes as C

    import torch

    dev = torch.device("cuda:0")
    t = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (rp, col, val, diag, b, x0)]
    it, rel = C.c_int32(), C.c_double()
    torch.cuda.synchronize()
    rc = entry(len(b), *(C.c_void_p(a.data_ptr()) for a in t[:5]), C.c_void_p(t[5].data_ptr()), rtol, max_iter, None,
               C.byref(it), C.byref(rel))
    torch.cuda.synchronize()
    return rc, t[5].cpu().numpy(), it.value, rel.value
