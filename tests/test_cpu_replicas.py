"""The multi-GPU form of the benchmark is N independent replicas (the solve has no
exchange between GPUs); its only collective is the max over ranks of the timed
region.  Checked here with two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seconds = 1.0 + rank          # rank 1 is the slow one
        t = bench.max_over_ranks(seconds, dist, "cpu")
        out[rank] = (t, bench.job_throughput(world, 10, t))
    finally:
        dist.destroy_process_group()


def test_two_replicas_max_over_ranks():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1] == (2.0, 10.0)


def test_single_rank_is_identity():
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.job_throughput(1, 4, 2.0) == 2.0
