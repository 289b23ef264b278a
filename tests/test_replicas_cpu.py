"""Replica aggregation of bench.py across ranks (gloo, world size 2, CPU): the
job's rate is computed from the slowest rank's time, identically on every
rank, as the multi-GPU benchmark computes it over NCCL."""

import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r took 100 + 50 r ms for 3 steps of 1,000 queries; e2e 2 + r s
        ms, value, e2e = bench.replica_throughput(100.0 + 50.0 * rank, 2.0 + rank, 1000, 3, 4,
                                                  world)
        out[rank] = (ms, value, e2e)
    finally:
        dist.destroy_process_group()


def test_replica_rate_uses_the_slowest_rank():
    world = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    slow_ms = 100.0 + 50.0 * (world - 1)
    slow_e2e = 2.0 + (world - 1)
    for r in range(world):
        ms, value, e2e = res[r]
        assert ms == pytest.approx(slow_ms)
        assert value == pytest.approx(world * 1000 * 3 / (slow_ms / 1000.0))
        assert e2e == pytest.approx(world * 1000 * 4 / slow_e2e)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    ms, value, e2e = bench.replica_throughput(200.0, 4.0, 500, 2, 2, 1)
    assert (ms, value, e2e) == (200.0, 500 * 2 / 0.2, 500 * 2 / 4.0)
