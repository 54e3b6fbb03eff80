"""The multi-GPU path of bench.py is N independent replicas: no collective on
the data path, only the reduction of per-rank units and times.  This runs that
reduction as two gloo ranks on CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r processed 1000 * (r + 1) units in (r + 1) * 0.5 s
        value, slowest = bench.replica_throughput(1000.0 * (rank + 1), 0.5 * (rank + 1), world, "cpu")
        rays = bench.reduce_over_ranks(10 + rank, world, "cpu", "sum")
        out[rank] = (value, slowest, rays)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_replica_reduction_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    for r in range(world):
        value, slowest, rays = out[r]
        assert slowest == pytest.approx(1.0)           # the slowest rank's time
        assert value == pytest.approx(3000.0 / 1.0)    # all units over that time
        assert rays == 21


def test_single_rank_is_identity():
    import bench

    value, slowest = bench.replica_throughput(500.0, 2.0, 1, "cpu")
    assert (value, slowest) == (250.0, 2.0)
