"""Replica path of bench.py on two gloo ranks (CPU): every rank takes the same
collective steps, the timing is the max over ranks, the whole-job throughput
counts every replica, and under torchrun the reference arm runs on rank 0
only."""
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


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    from datetime import timedelta
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        bench.rank_barrier(world)
        t = bench.max_over_ranks_on(100.0 + 50.0 * rank, world, torch.device("cpu"))
        v = bench.replica_throughput(world, 256, t)
        out[rank] = (t, v)
        bench.rank_barrier(world)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_replica_throughput_two_ranks():
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    for r in range(world):
        t, v = out[r]
        assert t == 150.0                       # the slowest rank's time, on every rank
        assert v == pytest.approx(2 * 256 / 0.150)  # all replicas' solves over that time


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks_on(12.5, 1, None) == 12.5
    assert bench.replica_throughput(1, 10, 1000.0) == 10.0


def test_reference_arm_runs_on_rank_zero_only():
    """A non-zero rank of the reference arm exits 0 without work or output."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
