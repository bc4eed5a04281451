"""Multi-process plumbing of bench.py, on CPU with the gloo backend.

The benchmarked path does not shard: each GPU solves its own system, so
bench.py --gpus N runs N independent replicas.  Its only cross-rank steps are a
barrier around the timed region and the max over ranks of the step time.
These tests run them as two real processes (world size 2) on 127.0.0.1, and
run the reference arm under torchrun, where rank 0 alone does the work and
prints the one JSON line.
"""
import json
import multiprocessing as mp
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    w, r, local, pg = bench.dist_init()
    try:
        bench.barrier(pg, local)
        got = bench.allmax(pg, 1.5 + r, local)   # rank 1 holds the larger time
        q.put((r, w, got))
    finally:
        pg.destroy_process_group()


def test_barrier_and_max_over_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == [(0, 2, 2.5), (1, 2, 2.5)]


def test_reference_arm_under_torchrun_prints_one_line():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), "bench.py", "--impl", "reference",
           "--gpus", "2", "--lattice", "4,4,4,8", "--steps", "1", "--warmup", "3", "--ref-sample-seconds",
           "0.2"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2
    assert d["value"] > 0 and d["e2e"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "port"
    fs = d["full_solve"]
    assert fs["converged"] and fs["true_rel_residual"] < 1e-9 and fs["iterations"] > 10
    for k in ("lattice", "volh", "sweeps", "plaquette", "parallelism"):
        assert k in d["config"]


def test_bench_launches_its_own_ranks():
    """bench.py --gpus 2 without torchrun starts two ranks itself; the line
    comes from rank 0 alone, with n_gpus 2 and the max over the ranks."""
    cmd = [sys.executable, "bench.py", "--gpus", "2", "--workload", "plumbing", "--steps", "2", "--warmup", "1"]
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2 and len(d["per_rank_s"]) == 2
    assert d["value"] == max(d["per_rank_s"]) and d["per_rank_s"][1] > 0.01
