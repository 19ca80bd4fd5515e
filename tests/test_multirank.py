"""The multi-rank plumbing of bench.py on CPU (gloo, world size 2).

The path does not shard: N GPUs run N independent replicas, and the only
cross-rank step is the max-over-ranks of the timings (a barrier and one
all-reduce).  These tests run that plumbing with two gloo ranks on the host:
the aggregate throughput uses the slowest rank's time, every rank takes the
same collective steps, and the reference arm runs on rank 0 only.
"""
import importlib.util
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    bench = load_bench()
    r, w, local = bench.dist_env()
    dist = bench.init_dist(w, local, "gloo")
    secs = 1.0 + rank  # rank 1 is the slow one
    slowest = bench.max_over_ranks(dist, secs, "cpu")
    sites, steps = 1000, 10
    value = sites * steps * w / slowest / 1e6
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, r, w, slowest, value))


def test_max_over_ranks_and_aggregate_throughput():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, r, w, slowest, value in res:
        assert r == rank and w == 2
        assert slowest == 2.0                         # the max over ranks, seen by every rank
        assert value == pytest.approx(1000 * 10 * 2 / 2.0 / 1e6)


def test_reference_arm_runs_on_rank_zero_only(tmp_path):
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "tgv64",
                        "--steps", "2", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""


def test_reference_arm_prints_one_line_on_rank_zero():
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "tgv64",
                        "--steps", "2", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if "unavailable" not in d:
        assert d["value"] > 0 and d["cpu_baseline"]["kind"] == "reference"
        assert d["e2e"]["h2d_bytes_per_step"] == 0
