"""Multi-GPU runs of the benchmark are independent replicas (the solve does
not shard: one grid per GPU).  Their only collective is the max-over-ranks of
the timings; this checks that step with two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = bench.max_over_ranks(1.0 + rank, dist, "cpu")  # rank 1 is the slow one
        out[rank] = (t, bench.replica_throughput(world, 1e6, t))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_replicas_take_the_slowest_rank():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 2.0
    assert res[0][1] == pytest.approx(1.0)  # 2 replicas x 1e6 points in 2 s = 1 Mpoints/s


def test_single_process_needs_no_collective():
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
