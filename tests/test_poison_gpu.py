"""Unwritten outputs: every output entry of the right-hand side is written.

The output buffer is filled with NaN before the launch (a race or a skipped partial tile
would leave NaN behind), on tiny and ragged meshes that exercise every halo, wrap and
partial-tile case of the 8 x 4 tiles: 2 x 2, 3 x 2, 8 x 6, 9 x 5, 17 x 3; periodic and
walls; all three arithmetic modes. The result must also equal the stateless host entry's.
"""
from __future__ import annotations

import numpy as np
import pytest

import sgnb
from cases import bump_case
from conftest import bits_equal

pytestmark = pytest.mark.gpu

MESHES = [(2, 2), (3, 2), (8, 6), (9, 5), (17, 3)]


@pytest.mark.parametrize("prec", [sgnb.FP64_EXACT, sgnb.FP64_FAST, sgnb.MIXED])
@pytest.mark.parametrize("bc", [0, 1])
@pytest.mark.parametrize("Nx,Ny", MESHES)
def test_rhs_writes_every_entry(prec, bc, Nx, Ny):
    import torch

    kw, U = bump_case(bc, Nx=Nx, Ny=Ny, Lx=1.25 * Nx, Ly=1.3 * Ny)
    with sgnb.SGN2DB200(precision=prec, **kw) as d:
        R = d.rhs(U)
        Ut = torch.from_numpy(U).cuda()
        out = torch.full_like(Ut, float("nan"))
        torch.cuda.synchronize()
        d.rhs_device(Ut.data_ptr(), out.data_ptr())
        _, sp = d.state_device_ptr()
        torch.cuda.ExternalStream(sp).synchronize()
        got = out.cpu().numpy()
        assert np.isfinite(got).all(), f"{np.isnan(got).sum()} entries left unwritten"
        assert bits_equal(got, R)
