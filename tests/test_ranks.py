"""The multi-process path of bench.py on the CPU: two gloo ranks.

Every rank runs an independent replica of the step; the job's time is the slowest
rank's, reduced with an all-reduce MAX.
"""

from __future__ import annotations

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


def _rank(rank, world, port, results):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    from datetime import timedelta

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=30))
    try:
        got = bench.max_over_ranks(10.0 * (rank + 1), dist, torch.device("cpu"))
        results[rank] = got
    finally:
        dist.destroy_process_group()


def test_time_is_the_slowest_ranks():
    world = 2
    port = _free_port()
    manager = mp.get_context("spawn").Manager()
    results = manager.dict()
    mp.start_processes(_rank, args=(world, port, results), nprocs=world, join=True,
                       start_method="spawn")
    assert dict(results) == {0: 20.0, 1: 20.0}


def test_single_process_needs_no_group():
    import bench

    assert bench.max_over_ranks(3.5, None, torch.device("cpu")) == 3.5
