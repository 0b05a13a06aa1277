"""The N > 1 path of bench.py on CPU: world size 2 over gloo (no GPU).

The step has no exchange between ranks (every rank is an independent replica); what crosses
ranks is the timing: the slowest rank's time and the sum of the units all ranks processed.
Also checks that the reference arm under torchrun prints one line, from rank 0."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r "took" 1.5 + r seconds for 1000 * (r + 1) particle-steps
        t, u = bench.reduce_over_ranks(dist, 1.5 + rank, 1000 * (rank + 1), device="cpu")
        # a second reduction in the same order on every rank (as the bench's graph form does)
        t2, u2 = bench.reduce_over_ranks(dist, 0.25 * (world - rank), 7, device="cpu")
        out.put((rank, t, u, t2, u2))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_timing_reduction_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, u, t2, u2 in res:
        assert t == 2.5 and u == 3000.0  # max of 1.5, 2.5; 1000 + 2000
        assert t2 == 0.5 and u2 == 14.0


def test_single_process_reduction_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.reduce_over_ranks(None, 1.25, 42) == (1.25, 42.0)


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libscdat_ref_omp.so")),
                    reason="reference library not built")
def test_reference_arm_under_torchrun_prints_once():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "3", "--warmup", "3", "--no-cpu-components",
           "--cpu-seconds", "1"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] in ("reference", "port")
    # rank 0 runs on all host threads, not the one thread torchrun gives each rank
    if d["cpu_baseline"]["kind"] == "reference":
        assert d["cpu_baseline"]["cores"] == (os.cpu_count() or 1)
