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


def test_bench_reads_its_denominators():
    """The roofline's inputs: the committed per-DOF DRAM traffic of the three kernel modes
    (profiles/traffic_per_dof.txt) and the HBM peak (MEASURED_PEAKS.json, else the stated
    fallback of 6650 GB/s)."""
    sys.path.insert(0, ROOT)
    import bench

    t = bench.traffic_per_dof()
    assert set(t) >= {"rhs", "stage", "fsal"}
    # measured DRAM bytes stay near the algorithmic 18.24 / 26.24 / 50.24 B/DOF
    for k, alg in (("rhs", 18.24), ("stage", 26.24), ("fsal", 50.24)):
        assert 0.8 * alg < t[k] < 1.2 * alg, (k, t[k])
    peak, kind = bench.measured_peak_hbm()
    assert kind in ("measured", "fallback") and peak > 1000.0


def test_reference_arm_other_ranks_do_nothing(monkeypatch, capsys):
    """Under torchrun only rank 0 runs the reference arm; the others exit without work."""
    sys.path.insert(0, ROOT)
    import argparse

    import bench

    monkeypatch.setenv("RANK", "1")
    bench.run_reference(argparse.Namespace(ref_device="cpu", steps=1, warmup=3, gpus=2))
    assert capsys.readouterr().out == ""


def test_cpu_baseline_loop_times_the_adaptive_loop():
    """The CPU baseline's loop leg runs the reference's integrateAdaptive (the compiled
    reference where it was built, else the oracle port) on a row strip of the
    configuration-2 mesh and reports DOF-updates/s over every right-hand side it took."""
    sys.path.insert(0, ROOT)
    import bench

    r = bench.cpu_baseline_loop(None, rows=2, span=0.2)
    assert r["value"] > 0 and r["cores"] == 1 and r["unit"] == bench.UNIT
    assert r["kind"] in ("reference", "port")
    assert "accepted" in r["sample"] and "2048x2" in r["sample"]
