"""The multi-rank bookkeeping of bench.py on CPU: two gloo ranks (the
replica runs use one process per GPU over NCCL with the same calls), each
with its own time; the reported rate is every rank's evaluations over the
slowest rank's time, and the reference arm runs on rank 0 only."""
import os
import socket
import subprocess
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        seconds = [2.0, 3.5][rank]        # this rank's timed region
        slowest = bench.reduce_max(seconds, dist, "cpu")
        q.put((rank, slowest, bench.replica_rate(world, 100, slowest)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replica_rate_takes_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    assert [o[1] for o in out] == [3.5, 3.5]
    assert all(abs(o[2] - 200 / 3.5) < 1e-12 for o in out)


def test_single_process_needs_no_group():
    assert bench.reduce_max(1.25, None, "cpu") == 1.25
    assert bench.replica_rate(1, 10, 2.0) == 5.0


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1"], env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0
    assert p.stdout.strip() == ""
