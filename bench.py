"""Benchmark: PIC particle-steps/s of the B200 PIC-MCC step (push + deposit + boundary +
MCC + Poisson solve + nodal field) on a synthetic Kuhn-box plasma, through the C ABI.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config NAME]

Workloads (all synthetic, seeded; the reference publishes no dataset):
  precision128  128^3 hex cells x 6 tets (12.4M tets outside the body), h = 1.6 m / 128, central 32^3-cell
                conducting body at -10 V, outer faces 0 V, electrons + H+ at n = 1e10 m^-3,
                Te = Ti = 1 eV, 64 particles per cell per species (~264M), dt = 2e-8 s,
                FP32 cell-relative push, fixed-point deposit, FP32-SpMV PCG under FP64
                refinement to 1e-10, elastic MCC (sigma 1e-19 m^2, n_n 1e14 m^-3), electrons
                re-sorted by tet every step (they cross ~0.7 cells per step), ions every 16
                [default]
  plain32       32^3 cells, h = 0.05 m, 8^3-cell body, 20 ppc, FP64, Jacobi-PCG to 1e-8
  batched64     64 independent scenarios stepped together (one launch per kernel over all of
                them, one CUDA-graph launch per step, launch shapes autotuned): box edge
                uniform in 16..64 cells of one Debye length, central body of a quarter of the
                edge at a bias uniform in -1000..-1 V, n log-uniform in 1e8..1e12 m^-3, Te and
                Ti log-uniform in 0.1..10 eV, 8..64 ppc per species, dt = 0.1 / omega_pe;
                mixed form, timed against the plain FP64 form of the same scenarios run one at
                a time
  surface256    256 x 256 x 128 cells of one Debye length (50M tets), a 32 x 32 x 16-cell body
                whose 6 faces are floating dielectric patches (eps_r 3, 1 mm) integrating their
                collected charge into FP64 potentials, n = 1e9 m^-3, Te = Ti = 5 eV, 16 ppc,
                dt = 0.1 / omega_pe; mixed form, with the FP64 form's face potentials after the
                same steps as the error reference
  surface_long  the same plasma and dielectric faces on a 64 x 64 x 32-cell box (8 x 8 x 4
                body) run for thousands of steps: the face-potential error of the mixed form
                against FP64 every 100 steps, beside FP64 controls (one velocity moved by one
                ulp, every velocity rounded to FP32, an independent seed) that size the
                run-to-run divergence of the chaotic particle dynamics
Every rank runs an independent replica ("replicas only": the path has no exchange step).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

QE, ME, MP = 1.602176634e-19, 9.1093837015e-31, 1.67262192369e-27

CONFIGS = {
    "precision128": dict(n=128, L=1.6, body=(48, 80), bias=-10.0, ppc=64, dt=2e-8, precision=1, rtol=1e-10,
                         density=1e10, te=1.0, ti=1.0, sort_interval=1, ion_sort_interval=16, precond="multigrid"),
    "plain32": dict(n=32, L=1.6, body=(12, 20), bias=-10.0, ppc=20, dt=2e-8, precision=0, rtol=1e-8, density=1e10,
                    te=1.0, ti=1.0, sort_interval=8),
    "batched64": dict(scenarios=64, seed=2026, precision=1, rtol=1e-10, sort_interval=4),
    "surface256": dict(cells=(256, 256, 128), body=((112, 144), (112, 144), (56, 72)), ppc=16, density=1e9, te=5.0,
                       ti=5.0, precision=1, rtol=1e-10, sort_interval=4, ion_sort_interval=16, eps_r=3.0,
                       thickness=1e-3),
    # the large surface-charging run's plasma and dielectric faces on a quarter-size box, run for
    # thousands of steps: the floating-potential error of the mixed form against FP64
    "surface_long": dict(cells=(64, 64, 32), body=((28, 36), (28, 36), (14, 18)), ppc=16, density=1e9, te=5.0,
                         ti=5.0, precision=1, rtol=1e-10, sort_interval=4, ion_sort_interval=16, eps_r=3.0,
                         thickness=1e-3),
}


def round_velocities_fp32(dom):
    """Round every particle velocity to FP32, as the precision form stores them: a perturbation
    of all particles at the level of the precision form's initial rounding, run in FP64."""
    for s in range(dom.nspecies):
        p = dom.get_particles(s)
        dom.set_particles(s, p["x"], p["v"].astype(np.float32).astype(np.float64), p["tet"], p["id"])


def nudge_one_velocity(dom, s=0):
    """Move one particle's x-velocity by one ulp (FP64) -- a perturbation at the level of the
    arithmetic's own rounding, to measure how far two runs of one form drift apart."""
    p = dom.get_particles(s)
    v = p["v"].copy()
    v[0, 0] = np.nextafter(v[0, 0], np.inf)
    dom.set_particles(s, p["x"], v, p["tet"], p["id"])


EPS0 = 8.8541878128e-12


def batched_scenarios(count, seed):
    """The seeded scenario list of the batched workload (sizes, plasma, bias, ppc, dt)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.integers(16, 65))
        dens = 10 ** rng.uniform(8, 12)
        te, ti = 10 ** rng.uniform(-1, 1), 10 ** rng.uniform(-1, 1)
        bias = rng.uniform(-1000, -1)
        ppc = int(rng.integers(8, 65))
        h = float(np.sqrt(EPS0 * te / (dens * QE)))  # one electron Debye length
        wpe = float(np.sqrt(dens * QE * QE / (EPS0 * ME)))
        q = max(1, n // 4)
        lo = (n - q) // 2
        out.append(dict(n=n, L=n * h, body=(lo, lo + q), bias=bias, ppc=ppc, dt=0.1 / wpe, density=dens, te=te,
                        ti=ti, rtol=1e-10, sort_interval=4))
    return out


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def reduce_over_ranks(dist, t_local, units, device="cuda"):
    """(the slowest rank's time, the units all ranks processed); every rank calls it, in the
    same order.  dist is torch.distributed (or None for one process)."""
    if dist is None:
        return t_local, float(units)
    import torch

    t = torch.tensor([t_local], device=device, dtype=torch.float64)
    u = torch.tensor([float(units)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t[0]), float(u[0])


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[4:8]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_domain(cfg, precision, capi, solve=True, mesh_cache=None):
    """A freshly seeded context of the workload (mesh arrays reused from mesh_cache)."""
    n = cfg["n"]
    h = cfg["L"] / n
    body = ((cfg["body"][0], cfg["body"][1]),) * 3 if cfg["body"] else None
    key = (n, cfg["L"], cfg["body"], cfg["bias"])
    if mesh_cache is not None and key in mesh_cache:
        m = mesh_cache[key]
    else:
        m = capi.kuhn_box_mesh((n, n, n), h, body=body, bias=cfg["bias"], wall=0.0)
        if mesh_cache is not None:
            mesh_cache[key] = m
    dom = capi.Domain(m["xyz"], m["tet"], m["dirichlet"], cfg["dt"], precision=precision, face_bc=(1,) * 6,
                      pcg_rtol=cfg["rtol"], pcg_max_iter=20000, sort_interval=cfg["sort_interval"])

    class Sp:
        def __init__(self, q, mass, w):
            self.q, self.m, self.w = q, mass, w

    w = cfg["density"] * h ** 3 / cfg["ppc"]
    dom.set_species([Sp(-QE, ME, w), Sp(QE, MP, w)])
    dom.seed_box(0, (n, n, n), h, body, cfg["ppc"], cfg["te"], 12345)
    dom.seed_box(1, (n, n, n), h, body, cfg["ppc"], cfg["ti"], 12345)
    if cfg.get("ion_sort_interval"):
        dom.set_species_sort_interval(1, cfg["ion_sort_interval"])
    for s in range(2):
        dom.set_elastic(s, 1e14, 1e-19, mode=2)  # null-collision MCC
    if cfg.get("precond") == "multigrid":
        dom.set_preconditioner(capi.PRECOND_MULTIGRID)
    dom.set_potential(m["phi"])
    if solve:
        dom.solve_field(allow_not_converged=True)
    return dom, m


def alg_bytes_push(dom, precision, particles):
    """Algorithmic bytes of one push launch (all species of a step): particle state read and
    written once (+ the 4-byte id the fused MCC reads), every tet record read once (FP64: the
    128-byte geometry record and the 96-byte nodal-E record; mixed: the first 128 bytes of its
    record), and each node's three 8-byte charge limbs read and written once per species."""
    b_p = 60 if precision == 1 else 108
    t_b = 128 if precision == 1 else 128 + 96
    n_b = 48 * dom.nspecies
    return particles * b_p + dom.T * t_b + dom.N * n_b


# DRAM bytes per stored particle of one step's push launches (all passes, both species; the
# electrons' pass 1 includes the gather of their re-sort): an ncu capture (dram__bytes_read.sum +
# dram__bytes_write.sum) of one step's six push launches on a 64^3-cell box at 64 ppc per species
# (31.9 M particles, 7.16 GB), divided by the particles; the full workload has the same density
# and access pattern.  None: not measured for the form.
PUSH_DRAM_BYTES_PER_PARTICLE = {1: 224.6, 0: None}


def cg_iteration_bytes(dom, precision):
    """Algorithmic bytes of one (inner) CG iteration of the field solve.  Jacobi: R rows x (15
    nonzeros x (value + column) + 7 vectors x 8 B).  Multigrid: the CG's own direction, mat-vec
    and update (3 + 3 + 6 vectors, the matrix once) plus one V-cycle, each level's arrays
    counted once per pass: a first sweep (3 vectors), three sweeps and a residual (matrix + 5
    vectors each), the restriction and prolongation (their weights and columns, the vectors they
    read and write), and on the coarsest level the dense inverse once."""
    V = 4 if precision == 1 else 8
    levels = dom.solver_levels()
    R0, nnz0, _ = levels[0]
    if len(levels) == 1:
        return R0 * (15 * V + 4 * 15 + 7 * 8)

    def csr_pass(R, nnz, vecs):
        return 4 * (R + 1) + nnz * (4 + V) + vecs * V * R

    b = 3 * V * R0 + csr_pass(R0, nnz0, 3) + 6 * V * R0
    for l in range(len(levels) - 1):
        R, nnz, t = levels[l]
        Rc = levels[l + 1][0]
        b += 3 * V * R + 4 * csr_pass(R, nnz, 5)
        b += 8 * t + 4 * (Rc + 1) + V * (R + Rc)          # restriction
        b += 8 * t + 4 * (R + 1) + V * (Rc + 2 * R)       # prolongation
    Rc, nc, _ = levels[-1]
    b += V * nc + 2 * V * Rc
    return b


def step_bytes(dom, precision, particles, pcg_iters):
    """Algorithmic bytes of one step by the per-step formula: particle state read and written
    (FP64 104 B, mixed 56 B), per-tet connectivity and geometry (112 B), per-node field, charge
    limbs and potential (48 B), and the (inner) CG iterations of the field solve."""
    b_p = 56 if precision == 1 else 104
    per_iter = cg_iteration_bytes(dom, precision)
    return particles * b_p + dom.T * 112 + dom.N * 48 + pcg_iters * per_iter, per_iter


def _timed_steps(torch, stream, step, steps, counter):
    """Times `steps` calls of step() with CUDA events on `stream`; counter() after each step
    gives its active particles.  Returns (ms, particle-steps, active particles per step)."""
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    ps, act = 0, []
    for _ in range(steps):
        step()
        a = counter()
        ps += a
        act.append(int(a))
    ev1.record(stream)
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1), ps, act


def run_ours(args, cfg):
    """Every form starts from its own freshly seeded context (the same seed, mesh and plasma),
    runs W untimed steps and then the same K timed steps, so the forms are compared on the
    same step indices and populations: the stepped context (the headline), the same workload as
    a one-scenario CUDA-graph batch, the plain FP64 form, and the end-to-end loop through the C
    ABI with host buffers."""
    import torch

    from scdat_b200 import build, capi

    build.build()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    prec = cfg["precision"]
    mesh_cache = {}
    # ---- the headline: stepped context (scdat_step per step) ----
    dom, mesh = build_domain(cfg, prec, capi, mesh_cache=mesh_cache)
    stream = torch.cuda.ExternalStream(dom.stream())
    for _ in range(args.warmup):
        dom.step(1)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    dom.set_timing(True)
    pcg_iters = []

    def count_headline():
        st = dom.stats()
        pcg_iters.append(st["last_pcg_iterations"])
        return st["active_particles"]

    ms, psteps, active = _timed_steps(torch, stream, lambda: dom.step(1), args.steps, count_headline)
    tm = dom.timing()
    clk = clocks.stop()
    phi_at = (args.warmup + args.steps, dom.fields()[1].copy())
    t_max, total_psteps = reduce_over_ranks(dist, ms / 1e3, psteps)
    value = total_psteps / t_max
    # roofline of the dominant kernel (the push), timed with events on the library stream
    push_ms = tm["push_ms"] / max(tm["push_launches"], 1)
    parts_per_launch = tm["push_particles"] / max(tm["push_launches"], 1)
    bytes_push = alg_bytes_push(dom, prec, parts_per_launch)
    peak, peak_kind = load_peaks()
    achieved = bytes_push / (push_ms / 1e3) / 1e9
    traffic = None
    if PUSH_DRAM_BYTES_PER_PARTICLE.get(prec) is not None:
        traffic = PUSH_DRAM_BYTES_PER_PARTICLE[prec] * parts_per_launch
    # the per-step formula over the whole step, and the field stage alone
    it_mean = float(np.mean(pcg_iters)) if pcg_iters else 0.0
    b_step, b_iter = step_bytes(dom, prec, psteps / max(args.steps, 1), it_mean)
    step_ms = t_max * 1e3 / args.steps
    field_ms = tm["field_ms"] / args.steps
    roof_step = {"alg_bytes": b_step, "achieved": b_step / (step_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                 "frac": b_step / (step_ms / 1e3) / 1e9 / peak, "peak_kind": peak_kind,
                 "formula": "P*b_p + T*112 + N*48 + I_pcg*(bytes of one CG iteration)", "cg_iteration_bytes": b_iter}
    roof_field = {"alg_bytes": it_mean * b_iter, "achieved": it_mean * b_iter / (field_ms / 1e3) / 1e9,
                  "peak": peak, "unit": "GB/s", "frac": it_mean * b_iter / (field_ms / 1e3) / 1e9 / peak,
                  "peak_kind": peak_kind, "kernel": "field stage (inner CG iterations, refinement, LSQ)",
                  "pcg_iterations_per_step_mean": it_mean, "levels": dom.solver_levels()}
    stored = int(sum(dom.count(s) for s in range(dom.nspecies)))
    dom.close()
    # ---- the same workload as a one-scenario batch (one CUDA-graph launch per step) ----
    graph = None
    if prec == 1 and args.graph_form:
        gdom, _ = build_domain(cfg, prec, capi, mesh_cache=mesh_cache)
        batch = capi.Batch([gdom])
        for _ in range(args.warmup):
            batch.step(1)
        gstream = torch.cuda.ExternalStream(batch.stream())
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        l0 = batch.kernel_launches()
        clocks = ClockSampler(local)
        clocks.start()
        gms, gps, gact = _timed_steps(torch, gstream, lambda: batch.step(1), args.steps,
                                      lambda: gdom.stats()["active_particles"])
        gclk = clocks.stop()
        g_max, g_total = reduce_over_ranks(dist, gms / 1e3, gps)
        graph = {"value": g_total / g_max, "unit": "particle-steps/s", "ms_per_step": g_max * 1e3 / args.steps,
                 "gpu_launches": int(batch.kernel_launches() - l0), "clocks": gclk, "active_per_step": gact,
                 "ratio_vs_stepped": (g_total / g_max) / value,
                 "form": "one CUDA-graph launch per step (one-scenario batch, Jacobi-PCG), fresh seeded context, "
                         "same steps"}
        batch.close()
        gdom.close()
    # ---- the plain FP64 form (the 1x of the mixed form's speed-up) ----
    fp64 = None
    if prec == 1 and args.fp64_compare:
        fdom, _ = build_domain(cfg, 0, capi, mesh_cache=mesh_cache)
        fstream = torch.cuda.ExternalStream(fdom.stream())
        for _ in range(args.warmup):
            fdom.step(1)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        fdom.set_timing(True)
        fms, fps, fact = _timed_steps(torch, fstream, lambda: fdom.step(1), args.steps,
                                      lambda: fdom.stats()["active_particles"])
        ftm = fdom.timing()
        f_max, f_total = reduce_over_ranks(dist, fms / 1e3, fps)
        p64 = fdom.fields()[1]
        err = float(np.abs(phi_at[1] - p64).max() / max(np.abs(p64).max(), 1e-300))
        fp64 = {"value": f_total / f_max, "unit": "particle-steps/s", "steps": args.steps,
                "ms_per_step": f_max * 1e3 / args.steps, "active_per_step": fact,
                "stage_ms_per_step": {"push": ftm["push_ms"] / args.steps, "field": ftm["field_ms"] / args.steps,
                                      "resort": ftm["sort_ms"] / args.steps},
                "ratio": value / (f_total / f_max),
                "phi_rel_err_vs_fp64": {"value": err, "after_steps": phi_at[0],
                                        "note": "both forms from the same seeded state over the same steps; "
                                                "relative to max |phi|"}}
        fdom.close()
    # ---- end to end through the C ABI with host buffers: per step, Dirichlet potentials in
    # from pinned host memory, then the ledger, statistics and the nodal potential back ----
    edom, _ = build_domain(cfg, prec, capi, mesh_cache=mesh_cache)
    dir_nodes = np.nonzero(mesh["dirichlet"])[0].astype(np.int64)
    h_nodes = torch.from_numpy(dir_nodes).pin_memory()
    h_vals = torch.from_numpy(mesh["phi"][dir_nodes].copy()).pin_memory()
    h_phi = torch.empty(edom.N, dtype=torch.float64).pin_memory()
    for _ in range(args.warmup):
        edom.step(1)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    e2e_ps = 0
    parts_s = np.zeros(3)  # host seconds: potentials in, step, results back
    for _ in range(args.steps):
        ta = time.perf_counter()
        edom.L.scdat_set_node_potentials(edom.h, len(dir_nodes), h_nodes.data_ptr(), h_vals.data_ptr())
        tb = time.perf_counter()
        edom.step(1)
        tc = time.perf_counter()
        edom.ledger()
        st = edom.stats()
        edom.L.scdat_get_fields(edom.h, None, h_phi.data_ptr(), None)
        parts_s += (tb - ta, tc - tb, time.perf_counter() - tc)
        e2e_ps += st["active_particles"]
    e_max, e_total = reduce_over_ranks(dist, time.perf_counter() - t0, e2e_ps)
    e2e_val = e_total / e_max
    h2d = len(dir_nodes) * 16
    d2h = edom.N * 8 + 7 * 8 * 8 + 120
    edom.close()
    out = {
        "metric": "PIC particle-steps/s on 1 B200 (mixed/batched vs plain FP64 at equal error)",
        "value": value,
        "unit": "particle-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": step_ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32" if prec == 1 else "f64",
        "data": "synthetic (seeded Kuhn-box plasma, no dataset)",
        "step_form": "scdat_step per step (stepped context)",
        "config": {"workload": args.config, "cells": cfg["n"] ** 3, "tets": dom.T, "nodes": dom.N,
                   "particles": stored, "ppc_per_species": cfg["ppc"],
                   "precision": "mixed" if prec == 1 else "fp64", "pcg_rtol": cfg["rtol"],
                   "preconditioner": cfg.get("precond", "jacobi"),
                   "pcg_iterations_per_step": pcg_iters, "active_per_step": active,
                   "l2": "inputs larger than L2 (particle state > 126 MB)", "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_kind": peak_kind, "kernel": "push (gather+boris+relocate+deposit+mcc)",
                     "alg_bytes_per_launch": bytes_push, "launch_ms": push_ms},
        "roofline_step": roof_step,
        "roofline_field": roof_field,
        "stage_ms_per_step": {"push": tm["push_ms"] / args.steps, "field": field_ms,
                              "resort": tm["sort_ms"] / args.steps},
        "gpu_launches": int(tm["kernel_launches"]),
        "clocks": clk,
        "e2e": {"value": e2e_val, "unit": "particle-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "host_ms_per_step": {"potentials_in": parts_s[0] * 1e3 / args.steps,
                                     "step": parts_s[1] * 1e3 / args.steps,
                                     "results_out": parts_s[2] * 1e3 / args.steps},
                "form": "fresh seeded context, W untimed steps, the same K steps timed with the host clock"},
    }
    if graph is not None:
        out["graph_form"] = graph
    if fp64 is not None:
        out["fp64_form"] = fp64
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(cfg, args)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


def run_batched(args, cfg):
    """The batched workload: the plain FP64 form one scenario at a time (the 1x), then the
    mixed form of the same scenarios as one batch (autotuned, CUDA graph), both for the same
    number of steps from the same seeded state; potentials compared at the end."""
    import torch

    from scdat_b200 import build, capi

    build.build()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=900))
    scen = batched_scenarios(args.scenarios or cfg["scenarios"], cfg["seed"])
    tune_steps = 6  # scdat_batch_autotune: 6 candidate shapes x 1 step
    total = tune_steps + args.warmup + args.steps
    # plain FP64 form, one scenario at a time
    fp64_ms, fp64_ps, phi64 = 0.0, 0, []
    for c in scen:
        dom, _ = build_domain(c, 0, capi)
        stream = torch.cuda.ExternalStream(dom.stream())
        for _ in range(total - args.steps):
            dom.step(1)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            dom.step(1)
            fp64_ps += dom.stats()["active_particles"]
        ev1.record(stream)
        torch.cuda.synchronize()
        fp64_ms += ev0.elapsed_time(ev1)
        phi64.append(dom.fields()[1])
        dom.close()
    # mixed form, all scenarios in one batch
    built = [build_domain(c, 1, capi) for c in scen]
    doms = [dm for dm, _ in built]
    batch = capi.Batch(doms)
    chosen = batch.autotune(1)
    for _ in range(args.warmup):
        batch.step(1)
    stream = torch.cuda.ExternalStream(batch.stream())
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches0 = batch.kernel_launches()
    clocks = ClockSampler(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    ps = 0
    for _ in range(args.steps):
        batch.step(1)
        ps += sum(d.stats()["active_particles"] for d in doms)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    launches = batch.kernel_launches() - launches0
    errs = []
    for d, p64 in zip(doms, phi64):
        errs.append(float(np.abs(d.fields()[1] - p64).max() / max(np.abs(p64).max(), 1e-300)))
    # controls on the worst scenario, each an FP64 run over the same steps against the FP64 run:
    # one velocity moved by one ulp (how far two FP64 runs drift apart on their own), and every
    # velocity rounded to FP32 (the precision form's initial rounding, FP64 arithmetic after it)
    kw = int(np.argmax(errs))
    worst = dict(index=kw, error=errs[kw], scenario={k: scen[kw][k] for k in ("n", "bias", "density", "te", "ti", "ppc")})
    for name, perturb in (("fp64_vs_fp64_nudged", nudge_one_velocity), ("fp64_vs_fp64_v32", round_velocities_fp32)):
        cdom, _ = build_domain(scen[kw], 0, capi)
        perturb(cdom)
        for _ in range(total):
            cdom.step(1)
        worst[name] = float(np.abs(cdom.fields()[1] - phi64[kw]).max() / max(np.abs(phi64[kw]).max(), 1e-300))
        cdom.close()
    parts = int(sum(d.count(s) for d in doms for s in range(d.nspecies)))
    # end to end through the C ABI with host buffers: per step, each scenario's Dirichlet
    # potentials in from pinned memory, the potentials and statistics back
    dirs = [np.nonzero(m["dirichlet"])[0].astype(np.int64) for _, m in built]
    h_nodes = [torch.from_numpy(dn).pin_memory() for dn in dirs]
    h_vals = [torch.from_numpy(m["phi"][dn].copy()).pin_memory() for (_, m), dn in zip(built, dirs)]
    h_phi = [torch.empty(d.N, dtype=torch.float64).pin_memory() for d in doms]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_ps = 0
    e2e_steps = max(1, min(args.steps, 10))
    for _ in range(e2e_steps):
        for d, hn, hv in zip(doms, h_nodes, h_vals):
            d.L.scdat_set_node_potentials(d.h, hn.shape[0], hn.data_ptr(), hv.data_ptr())
        batch.step(1)
        for d, hp in zip(doms, h_phi):
            d.L.scdat_get_fields(d.h, None, hp.data_ptr(), None)
            e2e_ps += d.stats()["active_particles"]
    e2e_val = e2e_ps / (time.perf_counter() - t0)
    h2d = int(sum(16 * len(dn) for dn in dirs))
    d2h = int(sum(8 * d.N + 120 for d in doms))
    batch.close()
    for d in doms:
        d.close()
    t_local = ms / 1e3
    t_max, total_ps = reduce_over_ranks(dist, t_local, ps)
    out = {
        "metric": "PIC particle-steps/s on 1 B200 (mixed/batched vs plain FP64 at equal error)",
        "value": total_ps / t_max,
        "unit": "particle-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_max * 1e3 / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded scenarios, no dataset)",
        "config": {"workload": "batched64", "scenarios": len(scen), "particles": parts,
                   "cells": int(sum(c["n"] ** 3 for c in scen)), "edge_cells": [c["n"] for c in scen],
                   "precision": "mixed, batched, CUDA graph", "tuning": chosen, "pcg_rtol": 1e-10,
                   "l2": "inputs larger than L2 (particle state > 126 MB)", "parallelism": f"replicas x{world}"},
        "fp64_form": {"value": fp64_ps / (fp64_ms / 1e3), "unit": "particle-steps/s", "steps": args.steps,
                      "ms_per_step": fp64_ms / args.steps, "note": "plain FP64 form, scenarios one at a time"},
        "phi_rel_err_vs_fp64": {"max": max(errs), "median": float(np.median(errs)), "after_steps": total,
                                "per_scenario": errs, "worst": worst},
        "gpu_launches": int(launches),
        "clocks": clk,
        "e2e": {"value": e2e_val, "unit": "particle-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
    }
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


def build_surface_domain(cfg, precision, capi, seed=4242):
    nx, ny, nz = cfg["cells"]
    h = float(np.sqrt(EPS0 * cfg["te"] / (cfg["density"] * QE)))
    dt = 0.1 / float(np.sqrt(cfg["density"] * QE * QE / (EPS0 * ME)))
    body = cfg["body"]
    m = capi.kuhn_box_mesh((nx, ny, nz), h, body=body, bias=0.0, wall=0.0)
    dom = capi.Domain(m["xyz"], m["tet"], m["dirichlet"], dt, precision=precision, face_bc=(1,) * 6,
                      pcg_rtol=cfg["rtol"], pcg_max_iter=20000, sort_interval=cfg["sort_interval"])

    class Sp:
        def __init__(self, q, mass, w):
            self.q, self.m, self.w = q, mass, w

    w = cfg["density"] * h ** 3 / cfg["ppc"]
    dom.set_species([Sp(-QE, ME, w), Sp(QE, MP, w)])
    dom.seed_box(0, (nx, ny, nz), h, body, cfg["ppc"], cfg["te"], seed)
    dom.seed_box(1, (nx, ny, nz), h, body, cfg["ppc"], cfg["ti"], seed)
    if cfg.get("ion_sort_interval"):
        dom.set_species_sort_interval(1, cfg["ion_sort_interval"])
    dom.set_potential(m["phi"])
    dom.set_surface_circuit(tuple(b[0] * h for b in body), tuple(b[1] * h for b in body), eps_r=cfg["eps_r"],
                            thickness=cfg["thickness"], v0=0.0)
    dom.solve_field(allow_not_converged=True)
    return dom, dt


def run_surface(args, cfg):
    """Large surface-charging run: the FP64 form first (its face potentials after W + K steps
    are the error reference and its K steps the 1x), then the mixed form on the same seeded
    state; value = the mixed form's particle-steps/s."""
    import torch

    from scdat_b200 import build, capi

    build.build()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=900))
    res = {}
    clk = None
    long_run = args.config == "surface_long"
    every = max(1, (args.warmup + args.steps) // 20)  # face-potential samples of the long run
    # (precision, control): the long run adds the FP64 form against itself with one velocity
    # nudged by an ulp, started from FP32-rounded velocities, and from an independent seed
    runs = [(0, None), (1, None)] + ([(0, "nudged"), (0, "v32"), (0, "seed")] if long_run else [])
    for prec, nudged in runs:
        dom, dt = build_surface_domain(cfg, prec, capi, seed=4243 if nudged == "seed" else 4242)
        if nudged == "nudged":
            nudge_one_velocity(dom)
        elif nudged == "v32":
            round_velocities_fp32(dom)
        stream = torch.cuda.ExternalStream(dom.stream())
        series = []
        for k in range(args.warmup):
            dom.step(1)
            if long_run and (k + 1) % every == 0:
                series.append(dom.surface_state()["V"].tolist())
        torch.cuda.synchronize()
        if prec == 1 and dist:
            dist.barrier()
        clocks = ClockSampler(local)
        if prec == 1:
            clocks.start()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        ps = 0
        for k in range(args.steps):
            dom.step(1)
            ps += dom.stats()["active_particles"]
            if long_run and (args.warmup + k + 1) % every == 0:
                series.append(dom.surface_state()["V"].tolist())
        ev1.record(stream)
        torch.cuda.synchronize()
        if prec == 1:
            clk = clocks.stop()
        ms = ev0.elapsed_time(ev1)
        srf = dom.surface_state()
        res[(prec, nudged)] = dict(ms=ms, ps=ps, V=srf["V"], Q=srf["Q"], series=series,
                                   particles=int(sum(dom.count(s) for s in range(2))), tets=dom.T, dt=dt,
                                   collected=int(np.asarray(srf["counts"]).sum()))
        dom.close()

    def rel(a, b):
        a, b = np.asarray(a), np.asarray(b)
        return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))

    r64, r32 = res[(0, None)], res[(1, None)]
    v64, v32 = r64["V"], r32["V"]
    err = rel(v32, v64)
    t_local = r32["ms"] / 1e3
    t_max, total_ps = reduce_over_ranks(dist, t_local, r32["ps"])
    fp = {"mixed_V": v32.tolist(), "fp64_V": v64.tolist(), "rel_err_vs_fp64": err,
          "after_steps": args.warmup + args.steps,
          "particles_collected": {"mixed": r32["collected"], "fp64": r64["collected"]}}
    if long_run:
        fp["series_every_steps"] = every
        fp["series_rel_err_vs_fp64"] = [rel(a, b) for a, b in zip(r32["series"], r64["series"])]
        for ctl in ("nudged", "v32", "seed"):
            rn = res[(0, ctl)]
            fp[f"fp64_{ctl}_vs_fp64"] = rel(rn["V"], v64)
            fp["particles_collected"][f"fp64_{ctl}"] = rn["collected"]
            fp[f"series_fp64_{ctl}_vs_fp64"] = [rel(a, b) for a, b in zip(rn["series"], r64["series"])]
        fp["series_fp64_mean_V"] = [float(np.mean(b)) for b in r64["series"]]
    out = {
        "metric": "PIC particle-steps/s on 1 B200 (mixed/batched vs plain FP64 at equal error)",
        "value": total_ps / t_max, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded, no dataset)",
        "config": {"workload": args.config, "cells": list(cfg["cells"]), "tets": r32["tets"],
                   "particles": r32["particles"], "dt": r32["dt"], "precision": "mixed",
                   "surface": "6 floating dielectric faces (eps_r 3, 1 mm), FP64 charge and potential",
                   "l2": "inputs larger than L2 (particle state > 126 MB)", "parallelism": f"replicas x{world}"},
        "fp64_form": {"value": r64["ps"] / (r64["ms"] / 1e3), "unit": "particle-steps/s",
                      "ms_per_step": r64["ms"] / args.steps},
        "floating_potential": fp,
        "clocks": clk,
    }
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


def reference_sample(cfg):
    """The reference particle path on a bounded sample of the workload: a 16^3-cell box of the
    same cell size, plasma and particles per cell, a 4^3-cell body at the same bias."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    n = 16
    h = cfg["L"] / cfg["n"]
    q = n // 4
    mesh = O.kuhn_box((n, n, n), h, body=((6, 6 + q), (6, 6 + q), (6, 6 + q)), bias=cfg["bias"])
    sp = O.plasma_species(cfg["density"], cfg["te"], cfg["ti"], h, cfg["ppc"])
    parts = O.seed_particles(mesh, sp, cfg["ppc"], 7)
    o = O.Oracle()
    A = o.assemble(mesh)
    phi, _, _ = o.poisson(mesh, A, np.zeros(mesh.N), mesh.phi_bc, rtol=1e-10)
    E = o.lsq(mesh, A, phi)
    return O, mesh, sp, parts, E


def cpu_baseline(cfg, args):
    O, mesh, sp, parts, E = reference_sample(cfg)
    P = parts["x"].shape[0]
    if O.reference_available(omp=True):
        ref = O.Reference(omp=True)
        total, steps, nt = 0.0, 0, 1
        cur = parts
        while total < args.cpu_seconds and steps < 20:
            out, secs, nt = ref.push_parallel(mesh, E, cur, sp, cfg["dt"])
            cur = dict(parts, x=out["x"], v=out["v"], tet=np.where(out["lost"] == 1, -1, out["tet"]))
            total += secs
            steps += 1
        ref.close()
        kind, sample = "reference", (f"reference CrossTetrahedron push+deposit (OpenMP branch structure, {nt} threads) "
                                     f"of {P} particles x {steps} steps on a 16^3-cell box at the workload's cell size, "
                                     f"plasma and ppc; field solve excluded (dense reference solve infeasible)")
    else:
        o = O.Oracle()
        t0 = time.perf_counter()
        steps = 0
        cur = parts
        while time.perf_counter() - t0 < args.cpu_seconds and steps < 20:
            out = o.push(mesh, E, cur, sp, cfg["dt"])
            cur = dict(parts, x=out["x"], v=out["v"], tet=np.where(out["lost"] == 1, -1, out["tet"]))
            steps += 1
        total = time.perf_counter() - t0
        nt = 1
        kind, sample = "port", (f"C oracle push+deposit (1 thread) of {P} particles x {steps} steps on a 16^3-cell "
                                f"box at the workload's cell size, plasma and ppc; field solve excluded")
    out = {"value": P * steps / total, "unit": "particle-steps/s", "cores": nt, "kind": kind, "sample": sample}
    if kind == "reference" and not args.no_cpu_components:
        out["components"] = cpu_components(O, cfg, mesh, sp, parts, E)
    return out


def cpu_components(O, cfg, mesh, sp, parts, E):
    """The other CPU figures of the path, each on a bounded sample (a few seconds apiece): the
    reference push as shipped (serial), the reference background MCC step, the Poisson solve by
    the CPU restatement (the reference's dense solve is infeasible at this size), and the full
    reference step (push, dense Poisson, field, statistics) on a 12^3-cell box."""
    comp = {}
    ref = O.Reference(omp=False)
    sub = {k: (v[:8192] if isinstance(v, np.ndarray) else v) for k, v in parts.items()}
    t0 = time.perf_counter()
    ref.push(mesh, E, sub, sp, cfg["dt"])
    dt_push = time.perf_counter() - t0
    comp["push_serial"] = {"value": 8192 / dt_push, "unit": "particle-steps/s", "cores": 1,
                           "sample": "reference CrossTetrahedron push+deposit as shipped (serial), 8192 particles x 1 step"}
    ve = parts["v"][parts["species"] == 0]
    t0 = time.perf_counter()
    ref.mcc_count(ve, 0, sp[0].w, 1e-19, 1e14, cfg["dt"], 7, 1)
    dt_mcc = time.perf_counter() - t0
    comp["mcc"] = {"value": ve.shape[0] / dt_mcc, "unit": "particles/s", "cores": 1,
                   "sample": f"reference MonteCarloCollisionHandler elastic step over {ve.shape[0]} electrons"}
    o = O.Oracle()
    A = o.assemble(mesh)
    rho = np.random.default_rng(5).normal(0.0, 1e-12, mesh.N)
    t0 = time.perf_counter()
    o.poisson(mesh, A, rho, mesh.phi_bc, rtol=1e-8)
    dt_pois = time.perf_counter() - t0
    comp["poisson_restatement"] = {"value": 1.0 / dt_pois, "unit": "solves/s", "cores": 1,
                                   "sample": f"C restatement Jacobi-PCG to 1e-8 on the {mesh.N}-node sample mesh"}
    n = 12
    h = cfg["L"] / cfg["n"]
    m12 = O.kuhn_box((n, n, n), h, body=((4, 8), (4, 8), (4, 8)), bias=cfg["bias"])
    sp12 = O.plasma_species(cfg["density"], cfg["te"], cfg["ti"], h, 2)
    p12 = O.seed_particles(m12, sp12, 2, 11)
    r = ref.cycle(m12, p12, sp12, 1, cfg["dt"], (1,) * 6, m12.phi_bc)
    ref.close()
    comp["full_step_12cubed"] = {"value": p12["x"].shape[0] / r["seconds"], "unit": "particle-steps/s",
                                 "seconds_per_step": r["seconds"], "cores": 1,
                                 "sample": f"reference PICCycle::executeTimeStep (dense Poisson on {m12.N} nodes) with "
                                           f"{p12['x'].shape[0]} particles, 1 step"}
    return comp


def run_reference(args, cfg):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # torchrun gives every rank one OpenMP thread; rank 0 alone runs the reference arm, on all
    # the host's threads (set before the reference library and its OpenMP runtime load)
    os.environ["OMP_NUM_THREADS"] = str(os.cpu_count() or 1)
    cb = cpu_baseline(cfg, args)
    out = {
        "impl": "reference",
        "metric": "PIC particle-steps/s on 1 B200 (mixed/batched vs plain FP64 at equal error)",
        "value": cb["value"],
        "unit": "particle-steps/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps,
        "warmup": args.warmup,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded Kuhn-box plasma, no dataset)",
        "config": {"workload": args.config, "sample": cb["sample"]},
        "cpu_baseline": cb,
        "e2e": {"value": cb["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="precision128", choices=sorted(CONFIGS))
    ap.add_argument("--n", type=int, default=0, help="override the number of cells per edge")
    ap.add_argument("--ppc", type=int, default=0, help="override particles per cell per species")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-cpu-components", action="store_true", help="CPU baseline without its component figures")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU baseline: seconds of reference push timed")
    ap.add_argument("--no-fp64-compare", dest="fp64_compare", action="store_false")
    ap.add_argument("--scenarios", type=int, default=0, help="batched64: number of scenarios (default 64)")
    ap.add_argument("--precond", choices=["jacobi", "multigrid"], default=None,
                    help="override the workload's field-solve preconditioner")
    ap.add_argument("--no-graph-form", dest="graph_form", action="store_false")
    args = ap.parse_args()
    cfg = dict(CONFIGS[args.config])
    if args.config in ("batched64", "surface256", "surface_long"):
        if args.impl == "reference":
            run_reference(args, dict(CONFIGS["precision128"]))
        elif args.config == "batched64":
            run_batched(args, cfg)
        else:
            run_surface(args, cfg)
        return
    if args.n:
        f = args.n / cfg["n"]
        cfg["body"] = (int(cfg["body"][0] * f), int(cfg["body"][1] * f))
        cfg["n"] = args.n
    if args.ppc:
        cfg["ppc"] = args.ppc
    if args.precond:
        cfg["precond"] = args.precond
    if args.impl == "reference":
        run_reference(args, cfg)
    else:
        run_ours(args, cfg)


if __name__ == "__main__":
    main()
