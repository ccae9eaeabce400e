"""Replica coordination over two ranks (gloo backend on CPU, 127.0.0.1): the timed
region's barrier, the maximum over ranks of each rank's device time, and the whole-job
rate = work of every replica / slowest replica's time."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from sympack_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        assert replicas.world_info() == (world, rank, rank)
        replicas.barrier(dist)
        # each rank "measured" different times; every rank must see the maxima
        mine = [10.0 + rank, 5.0 - rank, 7.5]
        got = replicas.max_over_ranks(mine, None, dist)
        out[rank] = got + [replicas.job_rate(100.0, world, got[0])]
        replicas.barrier(dist)
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_max_and_sum_the_work():
    world, port = 2, _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        assert res[rank][:3] == [11.0, 5.0, 7.5]
        assert res[rank][3] == pytest.approx(2 * 100.0 / 11e-3)


def test_single_process_without_group():
    assert replicas.max_over_ranks([3.0, 4.0]) == [3.0, 4.0]
    assert replicas.job_rate(10.0, 1, 1000.0) == pytest.approx(10.0)
