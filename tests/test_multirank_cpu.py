"""The bench's multi-rank plumbing on CPU: world size 2 over gloo (the
replicas' max-over-ranks time and summed work), and the reference arm under
torchrun, where rank 0 alone runs and prints one line."""
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


def _replica(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r timed 10 + r ms over 100 * (r + 1) edges
        ms, edges = bench.combine_replicas(10.0 + rank, 100 * (rank + 1), "cpu")
        e2e = bench.sum_over_ranks(1.5 * (rank + 1), "cpu")
        out.put((rank, ms, edges, e2e))
    finally:
        dist.destroy_process_group()


def test_replica_reduction_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_replica, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for _, ms, edges, e2e in got:
        assert ms == 11.0 and edges == 300.0 and e2e == 4.5


def test_reference_arm_under_torchrun_prints_once():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py",
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1",
           "--workload", "banded"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0
