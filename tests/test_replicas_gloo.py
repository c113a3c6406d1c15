"""Replica timing of bench.py across ranks (world_size 2, gloo on the CPU): every rank ends with the
slowest rank's time, and the whole-job value counts every replica's steps."""
import os
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, ws, port, out):
    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        elapsed = 100.0 + 25.0 * rank  # ms of this rank's K steps
        worst = bench.max_over_ranks(elapsed, dist)
        out[rank] = (worst, bench.replica_value(ws, 20, worst))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_world2():
    ws, port = 2, 29517
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(ws, port, out), nprocs=ws, join=True)
        res = dict(out)
    assert res[0] == res[1]
    worst, value = res[0]
    assert worst == pytest.approx(125.0)
    assert value == pytest.approx(2 * 20 / 0.125)


def test_single_process_value():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.5, None) == 3.5
    assert bench.replica_value(1, 20, 100.0) == pytest.approx(200.0)
