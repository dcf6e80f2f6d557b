"""Host logic of the x-slab decomposition: the column split, the neighbour links, and the
distributed edge exchange and partial gather run as gloo ranks on the CPU (the same
torch.distributed calls the solver makes over NCCL between GPUs)."""
from __future__ import annotations

import os
import socket
import types

import pytest
import torch.multiprocessing as mp

from sgnb.slabs import LocalExchange, neighbours, slab_partition, tile_count


def test_partition_rule():
    # the first Nx % size slabs take one column more (src/parallel/slab1d.h:55-72)
    assert [slab_partition(10, 3, r) for r in range(3)] == [(0, 4), (4, 3), (7, 3)]
    assert [slab_partition(12, 4, r) for r in range(4)] == [(0, 3), (3, 3), (6, 3), (9, 3)]
    for Nx in (1, 7, 64, 513):
        for size in range(1, min(Nx, 9) + 1):
            parts = [slab_partition(Nx, size, r) for r in range(size)]
            assert parts[0][0] == 0 and sum(w for _, w in parts) == Nx
            assert all(parts[r][0] + parts[r][1] == parts[r + 1][0] for r in range(size - 1))
            assert max(w for _, w in parts) - min(w for _, w in parts) <= 1
    with pytest.raises(ValueError):
        slab_partition(2, 3, 0)
    with pytest.raises(ValueError):
        slab_partition(8, 2, 2)


def test_neighbours_and_tiles():
    assert neighbours(0, 1, True) == (0, 0)
    assert neighbours(0, 1, False) == (None, None)
    assert [neighbours(r, 3, True) for r in range(3)] == [(2, 1), (0, 2), (1, 0)]
    assert [neighbours(r, 3, False) for r in range(3)] == [(None, 1), (0, 2), (1, None)]
    assert tile_count(8, 4) == 1 and tile_count(9, 5) == 4 and tile_count(512, 512) == 8192


def _fake_slab(torch, rank, Ny=3):
    n = 5 * Ny * 5
    return types.SimpleNamespace(
        sendL=torch.full((n,), 10.0 * rank + 1, dtype=torch.float64),
        sendR=torch.full((n,), 10.0 * rank + 2, dtype=torch.float64),
        ghostL=torch.zeros(n, dtype=torch.float64),
        ghostR=torch.zeros(n, dtype=torch.float64),
        nblk=rank + 1,
        partials=torch.arange(3 * (rank + 1), dtype=torch.float64) + 100.0 * rank)


def _check_edges(slabs_by_rank, size, periodic, ghosts):
    for r in range(size):
        left, right = neighbours(r, size, periodic)
        gL, gR = ghosts[r]
        assert gL == (0.0 if left is None else 10.0 * left + 2)
        assert gR == (0.0 if right is None else 10.0 * right + 1)


def test_local_exchange_links():
    import torch

    for size, periodic in ((1, True), (1, False), (3, True), (3, False), (4, True)):
        slabs = [_fake_slab(torch, r) for r in range(size)]
        ex = LocalExchange(size, periodic)
        ex.edges(slabs)
        ghosts = {r: (float(s.ghostL[0]), float(s.ghostR[0])) for r, s in enumerate(slabs)}
        _check_edges(slabs, size, periodic, ghosts)
        allp, nblk = ex.gather(slabs, torch)
        mb = size
        assert nblk == mb * size and allp.numel() == 3 * nblk
        for r, s in enumerate(slabs):
            seg = allp[3 * mb * r: 3 * mb * (r + 1)]
            assert torch.equal(seg[: 3 * s.nblk], s.partials)
            assert torch.count_nonzero(seg[3 * s.nblk:]) == 0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    from sgnb.slabs import DistExchange

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    res = {}
    for periodic in (True, False):
        slab = _fake_slab(torch, rank)
        ex = DistExchange(periodic)
        ex.edges([slab])
        allp, nblk = ex.gather([slab], torch)
        res[periodic] = (float(slab.ghostL[0]), float(slab.ghostR[0]),
                         bool(torch.all(slab.ghostL == slab.ghostL[0])),
                         bool(torch.all(slab.ghostR == slab.ghostR[0])),
                         allp.tolist(), nblk)
    out[rank] = res
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_dist_exchange_gloo(world):
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn")
    import torch

    for periodic in (True, False):
        ghosts = {r: out[r][periodic][:2] for r in range(world)}
        assert all(out[r][periodic][2] and out[r][periodic][3] for r in range(world))
        _check_edges(None, world, periodic, ghosts)
        mb = world  # the largest block count (rank + 1)
        for r in range(world):
            allp, nblk = out[r][periodic][4], out[r][periodic][5]
            assert nblk == mb * world
            for q in range(world):
                seg = allp[3 * mb * q: 3 * mb * (q + 1)]
                want = (torch.arange(3 * (q + 1), dtype=torch.float64) + 100.0 * q).tolist()
                assert seg[: 3 * (q + 1)] == want and not any(seg[3 * (q + 1):])


def _slab_statics(kind, par, bc, Nx, Ny, Lx, Ly, ex0, nx):
    import ctypes as C

    import numpy as np

    import sgnb

    h = sgnb._DescHolder(4, nx, Ny, Lx, Ly, 9.81, 0.0, 1.5, 0.0, bc, bc, sgnb.FP64_EXACT, 0,
                         kind, par, None, None)
    h.desc.Nx_global, h.desc.ex_offset = Nx, ex0
    Nd, nf = 25 * nx * Ny, 5 * nx * Ny
    out = dict(Hnod=np.zeros(Nd), Hx=np.zeros(Nd), Hy=np.zeros(Nd), HfaceX=np.zeros(nf),
               HfaceY=np.zeros(nf), HfaceXEnd=np.zeros(5 * Ny), HfaceYEnd=np.zeros(5 * nx))
    rc = sgnb.lib().sgnb_setup_bathymetry(C.byref(h.desc), *(sgnb._ptr(out[k]) for k in (
        "Hnod", "Hx", "Hy", "HfaceX", "HfaceY", "HfaceXEnd", "HfaceYEnd")))
    return rc, out


@pytest.mark.parametrize("bc", [0, 1])
def test_slab_bathymetry_is_the_whole_mesh_columns(bc):
    """A slab's statics are its columns of the whole mesh's; across its right edge it sees
    the next column's left faces (x = 0 at the periodic wrap)."""
    import numpy as np

    import sgnb

    Nx, Ny, Lx, Ly = 11, 5, 5.5, 3.0
    kind, par = sgnb.BATHY_SHOAL, (1.0, 0.6, 0.3 * Lx, 0.45 * Ly, 0.25 * Lx, 0.2 * Ly)
    full = sgnb.setup_bathymetry(P=4, Nx=Nx, Ny=Ny, Lx=Lx, Ly=Ly, bathy_kind=kind,
                                 bathy_par=par, bc_x=bc, bc_y=bc)
    cols = lambda a, k, a0, w: a.reshape(Ny, Nx, k)[:, a0:a0 + w, :].reshape(-1)  # noqa: E731
    for a0, w in (slab_partition(Nx, 3, r) for r in range(3)):
        rc, s = _slab_statics(kind, par, bc, Nx, Ny, Lx, Ly, a0, w)
        assert rc == 0
        for k in ("Hnod", "Hx", "Hy"):
            assert np.array_equal(s[k], cols(full[k], 25, a0, w)), k
        for k in ("HfaceX", "HfaceY"):
            assert np.array_equal(s[k], cols(full[k], 5, a0, w)), k
        assert np.array_equal(s["HfaceYEnd"], full["HfaceYEnd"][5 * a0: 5 * (a0 + w)])
        if a0 + w < Nx:
            want = full["HfaceX"].reshape(Ny, Nx, 5)[:, a0 + w, :].reshape(-1)
        elif bc == 0:
            want = full["HfaceX"].reshape(Ny, Nx, 5)[:, 0, :].reshape(-1)
        else:
            want = full["HfaceXEnd"]
        assert np.array_equal(s["HfaceXEnd"], want)
    # the desc check: 0 <= ex_offset, ex_offset + Nx <= Nx_global
    assert _slab_statics(kind, par, bc, Nx, Ny, Lx, Ly, 9, 3)[0] == 1
    assert _slab_statics(kind, par, bc, Nx, Ny, Lx, Ly, -1, 3)[0] == 1
