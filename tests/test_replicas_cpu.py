"""Replica timing of bench.py on two CPU ranks (gloo): every rank learns the
slowest rank's step time, and the job value counts every rank's bytes over
that time (the N > 1 path, which runs independent replicas with no
data-path collective)."""
import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms_local = [1.5, 4.0][rank]
        allmax = lambda v: bench.max_over_ranks(v, world, torch, dist, "cpu")  # noqa: E731
        ms, value = bench.replica_value(ms_local, 1.0e9, world, allmax)
        out[rank] = (ms, value)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_replica_value_uses_the_slowest_rank():
    world = 2
    port = 29500 + (os.getpid() % 1000)
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1]
    ms, value = res[0]
    assert ms == 4.0
    assert value == pytest.approx(2 * 1.0e9 / 4.0e-3 / 1e9)   # 500 GB/s


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    ms, value = bench.replica_value(2.0, 1.0e9, 1, lambda v: v)
    assert ms == 2.0 and value == pytest.approx(500.0)
