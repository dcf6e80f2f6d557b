"""Multi-GPU layout of the benchmark: independent replicas, one per rank, no data-path
collective. The host-side aggregation (max time over ranks, summed work) runs here as two
gloo ranks on the CPU."""
from __future__ import annotations

import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    times = [1.0 + rank, 2.0 * (rank + 1)]
    works = [100.0 * (rank + 1), 7.0]
    t, w = bench.reduce_over_ranks(times, works, dist, "cpu")
    out[rank] = (t, w)
    dist.barrier()
    dist.destroy_process_group()


def test_replica_aggregation_two_ranks():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn")
    for r in range(world):
        t, w = out[r]
        assert t == [2.0, 4.0]          # slowest rank
        assert w == [300.0, 14.0]       # all ranks' work


def test_single_process_passthrough():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.reduce_over_ranks([1.5, 2.5], [3.0, 4.0], None, "cpu") == ([1.5, 2.5], [3.0, 4.0])
