"""The bench's multi-rank logic (replicas, max-over-ranks timing, whole-job
value) on two CPU ranks with the gloo backend."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = 1.0 + rank * 2.5              # rank 1 is the slow one
        t = bench.max_over_ranks(mine, dist)
        out[rank] = t
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0] == out[1] == 3.5


def test_job_value_and_single_rank():
    assert bench.max_over_ranks(2.0, None) == 2.0
    # two replicas of 10 products of 1 GB each in 0.5 s -> 40 GB/s whole job
    assert bench.job_value(10 * 1e9, 2, 0.5) / 1e9 == pytest.approx(40.0)
