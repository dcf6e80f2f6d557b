"""Runs every fused FP64 kernel family of the range-checked build (libsgnb_checked.so) on
ragged meshes and prints the out-of-range access count as the last line ("oob N").

Started by tests/test_checked_gpu.py in its own process with SGNB_LIBRARY=checked, so that
this process loads the checked library instead of the normal one. Covers the right-hand
side and the BS3(2) stages (exact, fast and mixed modes, periodic and walls, partial tiles,
Manning friction), Gauss-Legendre points (trace pre-pass and GAUSS variant), the batched kernels in
every tile shape and grid form (mixed batches too), slab edges (ghost reads, fused edge writes, packs), and the adjoint (right-hand-side VJP, gauge
trajectory and its VJP with checkpoints).
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "sgn-hyperbolic-gpu_b200"))
sys.path.insert(0, HERE)

import sgnb  # noqa: E402
from cases import ALPHA, GAMMA, G, bump_case, gauss_case, gll5, make_state, node_coords  # noqa: E402
from sgnb.slabs import PeerSlabSolver, SlabSolver  # noqa: E402

MESHES = [(2, 2), (3, 2), (8, 6), (9, 5), (17, 3), (13, 11)]


def count(reset=False):
    n = C.c_longlong()
    rc = sgnb.lib().sgnb_checked_oob(0, C.byref(n), int(reset))
    if rc != 0:
        raise SystemExit("not the checked build")
    return n.value


def main():
    assert os.path.basename(sgnb.LIB_PATH) == "libsgnb_checked.so", sgnb.LIB_PATH
    count(reset=True)
    for Nx, Ny in MESHES:
        for bc in (0, 1):
            kw, U = bump_case(bc, Nx=Nx, Ny=Ny, Lx=1.25 * Nx, Ly=1.3 * Ny)
            for prec in (sgnb.FP64_EXACT, sgnb.FP64_FAST, sgnb.MIXED):
                for n_man in (0.0, 0.03):
                    with sgnb.SGN2DB200(precision=prec, **dict(kw, nManning=n_man)) as d:
                        d.rhs(U)
                        d.upload(U)
                        d.integrate_steps(0.0, d.cfl_time_step(0.4), 3)
                        if prec != sgnb.MIXED:
                            d.rk4_steps(0.0, [d.cfl_time_step(0.4)] * 2)
            gk, GU = gauss_case(bc, Nx=Nx, Ny=Ny, Lx=1.25 * Nx, Ly=1.3 * Ny)
            with sgnb.SGN2DB200(precision=sgnb.FP64_FAST, **gk) as d:
                d.rhs(GU)
                d.upload(GU)
                d.integrate_steps(0.0, d.cfl_time_step(0.4), 2)
                d.rk4_steps(0.0, [d.cfl_time_step(0.4)])
    # batches: every tile shape, one CTA per tile and persistent grids
    insts = []
    for i, (Nx, Ny) in enumerate(MESHES):
        kw, _ = bump_case(i % 2, Nx=Nx, Ny=Ny, Lx=1.25 * Nx, Ly=1.3 * Ny)
        kw = dict(kw)
        kw.pop("P")
        insts.append(kw)
    b = sgnb.SGNBatch(insts)
    for shape in (0, 1, 2):
        for blocks in (0, 148):
            for i, kw in enumerate(insts):
                _, U = bump_case(i % 2, Nx=kw["Nx"], Ny=kw["Ny"], Lx=kw["Lx"], Ly=kw["Ly"])
                b[i].upload(U)
            b.config = (shape, blocks)
            b.integrate_steps(np.full(len(insts), 1e-3), 2)
    b.close()
    bm = sgnb.SGNBatch(insts, precision=sgnb.MIXED)
    for blocks in (0, 148):
        for i, kw in enumerate(insts):
            _, U = bump_case(i % 2, Nx=kw["Nx"], Ny=kw["Ny"], Lx=kw["Lx"], Ly=kw["Ly"])
            bm[i].upload(U)
        bm.config = (0, blocks)
        bm.integrate_steps(np.full(len(insts), 1e-3), 2)
    bm.close()
    # slabs: ghost reads, packs, fused edge writes, controllers on all slabs' partials
    for bc in (0, 1):
        kw, U = bump_case(bc, Nx=13, Ny=5, Lx=6.5, Ly=4.0)
        kw = dict(kw, precision=sgnb.FP64_FAST)
        with SlabSolver(kw, nslabs=3) as s:
            s.rhs(U)
            s.upload(U)
            s.integrate_steps(0.0, 1e-3, 3)
        with PeerSlabSolver(kw, nslabs=3, streams="per-slab") as s:
            s.rhs(U)
            s.upload(U)
            s.integrate_steps(0.0, 1e-3, 3)
    # the adjoint: one right-hand side's VJP, and a checkpointed gauge trajectory with its
    # VJP (cell-mean bathymetry), periodic and walls, with and without friction
    from sgnb import adjoint as ADJ

    for bc in (0, 1):
        kw, U = bump_case(bc, Nx=9, Ny=5, Lx=9.0, Ly=5.0)
        for n_man in (0.0, 0.03):
            with sgnb.SGN2DB200(precision=sgnb.FP64_FAST, **dict(kw, nManning=n_man)) as d:
                d.rhs_vjp(U, np.linspace(-1.0, 1.0, U.size))
        Nx, Ny, Lx, Ly = 7, 5, 7.0, 5.0
        means = np.linspace(0.8, 1.0, Nx * Ny)
        ak = dict(P=4, Nx=Nx, Ny=Ny, Lx=Lx, Ly=Ly, g=G, c=ALPHA * np.sqrt(G), gamma=GAMMA,
                  bc_x=bc, bc_y=bc, bathy_kind=sgnb.BATHY_CELLS,
                  bathy_par=np.concatenate([[Nx, Ny, Lx, Ly], means]))
        x, y = node_coords(4, Nx, Ny, Lx, Ly, gll5())
        eta0 = 0.03 * np.exp(-((x - 3.0) ** 2 + (y - 2.0) ** 2))
        with sgnb.SGN2DB200(precision=sgnb.FP64_FAST, **ak) as d:
            H = sgnb.setup_bathymetry(**{k: ak[k] for k in ("P", "Nx", "Ny", "Lx", "Ly", "bc_x",
                                                             "bc_y", "bathy_kind", "bathy_par")})["Hnod"]
            z = np.zeros_like(H)
            d.upload(make_state(H + eta0, z, z, z, z))
            dts = np.full(9, 0.4 * d.cfl_time_step(0.5))
            with ADJ.SGNAdjoint(d, dts, np.array([0, 40, 300, H.size - 1]), checkpoint_every=4) as A:
                eta = A.forward(means, eta0)
                A.vjp(np.ones_like(eta))
    print(f"oob {count()}")


if __name__ == "__main__":
    main()
