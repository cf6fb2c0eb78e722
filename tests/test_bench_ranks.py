"""The bench's multi-rank bookkeeping on CPU: two gloo ranks (replicas) agree
on the slowest rank's time, and the whole-job figure counts every rank's
points over that time."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank  # rank 1 is the slow replica
        out[rank] = bench.max_over_ranks(dist, ms, device="cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        got = dict(out)
    assert got == {0: 15.0, 1: 15.0}


def test_job_throughput_counts_every_rank():
    assert bench.max_over_ranks(None, 12.5) == 12.5
    one = bench.job_gpts(1, 1_000_000_000, 10, 20.0)
    assert one == pytest.approx(500.0)
    assert bench.job_gpts(4, 1_000_000_000, 10, 20.0) == pytest.approx(4 * one)
