"""sgnb_diag_noalloc, the allocation-free diagnostics entry point, against the context's
own sgnb_max_wave_speed / sgnb_mass / sgnb_energy.

It exists for callers that cannot allocate device memory (a framework owning all of it
through its own pool, or a fixed-budget time loop that must not call cudaMalloc between
steps): it keeps its per-block partials in a library-owned __device__ array. Two calls in
a row must both agree with the context path (the array keeps the previous call's
contents), within the tolerances of tests/test_rhs_gpu.py::test_diagnostics. This file is
collected last so that a failure here cannot hide earlier ones.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import sgnb
from cases import bump_case

pytestmark = pytest.mark.gpu


def _call(what, kw, U_ptr, H_ptr, out_ptr):
    return sgnb.lib().sgnb_diag_noalloc(what, kw["Nx"], kw["Ny"], kw["Lx"], kw["Ly"], kw["g"],
                                        kw["c"], kw["gamma"], C.c_void_p(U_ptr),
                                        C.c_void_p(H_ptr), C.c_void_p(out_ptr), None)


@pytest.mark.parametrize("Nx,Ny,bc", [(8, 6, 0), (33, 17, 1), (181, 93, 0)])
def test_noalloc_diagnostics_match_context(Nx, Ny, bc):
    import torch

    kw, U = bump_case(bc, Nx=Nx, Ny=Ny)
    H = sgnb.setup_bathymetry(Nx=Nx, Ny=Ny, Lx=kw["Lx"], Ly=kw["Ly"], bathy_kind=kw["bathy_kind"],
                              bathy_par=kw["bathy_par"], bc_x=bc, bc_y=bc)["Hnod"]
    with sgnb.SGN2DB200(precision=sgnb.FP64_EXACT, **kw) as d:
        d.upload(U)
        ref = {0: d.max_wave_speed(), 1: d.mass(), 2: d.energy()}
    Ut = torch.from_numpy(U).cuda()
    Ht = torch.from_numpy(H).cuda()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    for _ in range(2):  # two calls in a row share the scratch array
        for what in (0, 1, 2):
            out.fill_(np.nan)
            torch.cuda.synchronize()
            assert _call(what, kw, Ut.data_ptr(), Ht.data_ptr(), out.data_ptr()) == 0
            torch.cuda.synchronize()
            got = out.item()
            if what == 0:
                assert got == ref[0]
            else:
                assert got == pytest.approx(ref[what], rel=1e-13)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    kw, _ = bump_case()
    x = torch.zeros(5, dtype=torch.float64, device="cuda")
    kw = dict(kw, Nx=2048, Ny=1311)  # 25 * 2048 * 1311 > 67,108,864 nodes
    assert _call(1, kw, x.data_ptr(), x.data_ptr(), x.data_ptr()) == 1
    kw = dict(kw, Nx=2048, Ny=1310)  # fits; not launched here (x is too small)
    assert 25 * 2048 * 1310 <= 67108864


def test_noalloc_largest_accepted_mesh():
    """The largest mesh the scratch array takes (2048 x 1310: 67,072,000 nodes per field,
    16,375 of the 16,384 partial slots, the final pass folding 64 partials per thread):
    the mass of a seeded depth field equals the quadrature-weighted sum formed by torch,
    on two calls in a row."""
    import torch

    Nx, Ny, Lx, Ly = 2048, 1310, 40.0, 26.0
    Nd = 25 * Nx * Ny
    assert (Nd + 4095) // 4096 <= 16384
    kw = dict(Nx=Nx, Ny=Ny, Lx=Lx, Ly=Ly, g=9.81, c=3.0 * np.sqrt(9.81), gamma=1.5)
    g = torch.Generator(device="cuda").manual_seed(5)
    U = torch.zeros(5 * Nd, dtype=torch.float64, device="cuda")
    U[:Nd] = 0.45 + 0.05 * torch.rand(Nd, generator=g, dtype=torch.float64, device="cuda")
    qw = torch.tensor(sgnb.fr_tables()["qw"], dtype=torch.float64, device="cuda")
    w = (qw[None, :] * qw[:, None]).reshape(25).repeat(Nx * Ny)  # node a + 5 b
    ref = float((w * U[:Nd]).sum()) * (0.5 * Lx / Nx) * (0.5 * Ly / Ny)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    for _ in range(2):
        out.fill_(np.nan)
        torch.cuda.synchronize()
        assert _call(1, kw, U.data_ptr(), U.data_ptr(), out.data_ptr()) == 0
        torch.cuda.synchronize()
        assert out.item() == pytest.approx(ref, rel=1e-12)
