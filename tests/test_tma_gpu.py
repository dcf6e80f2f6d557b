"""Tile loads by the tensor-memory accelerator against the per-thread copies.

On meshes that are a whole number of 8x4 tiles the stage kernels take their own-node
tiles (state or stage derivatives, nodal depths) by TMA copies described by tensor maps of
the context's buffers; SGNB_TMA=0 at context creation keeps the per-thread asynchronous
copies. Only the data movement differs, so adaptive runs must take the same steps and
end in the same bits, in every arithmetic mode and with periodic and wall boundaries.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

import sgnb
from cases import bump_case

pytestmark = pytest.mark.gpu


def run(prec, kw, U, steps, tma):
    old = os.environ.get("SGNB_TMA")
    os.environ["SGNB_TMA"] = "1" if tma else "0"
    try:
        with sgnb.SGN2DB200(precision=prec, **kw) as d:
            d.upload(U)
            dt0 = d.cfl_time_step(0.5)
            st = d.integrate_steps(0.0, dt0, steps)
            return d.download(), (st.accepted, st.rejected, st.rhsEvals)
    finally:
        if old is None:
            del os.environ["SGNB_TMA"]
        else:
            os.environ["SGNB_TMA"] = old


@pytest.mark.parametrize("prec", [sgnb.FP64_EXACT, sgnb.FP64_FAST, sgnb.MIXED])
@pytest.mark.parametrize("bc", [0, 1])
def test_tile_copies_bitwise(prec, bc):
    kw, U = bump_case(bc, Nx=24, Ny=16, Lx=12.0, Ly=8.0)  # 3 x 4 whole tiles
    a, sa = run(prec, kw, U, 8, True)
    b, sb = run(prec, kw, U, 8, False)
    assert sa == sb and sa[0] == 8
    assert np.isfinite(a).all()
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


def rhs_pair(prec, kw, U, tma):
    old = os.environ.get("SGNB_TMA")
    os.environ["SGNB_TMA"] = "1" if tma else "0"
    try:
        with sgnb.SGN2DB200(precision=prec, **kw) as d:
            d.upload(U)
            a = d.rhs_once()  # input: the context's state buffer
            b = d.rhs(U)      # input: the context's scratch (host round trip)
            return a, b
    finally:
        if old is None:
            del os.environ["SGNB_TMA"]
        else:
            os.environ["SGNB_TMA"] = old


@pytest.mark.parametrize("prec", [sgnb.FP64_EXACT, sgnb.FP64_FAST])
def test_rhs_tile_copies_bitwise(prec):
    """The right-hand-side mode with its input's map encoded per launch."""
    kw, U = bump_case(1, Nx=24, Ny=16, Lx=12.0, Ly=8.0)
    a1, b1 = rhs_pair(prec, kw, U, True)
    a0, b0 = rhs_pair(prec, kw, U, False)
    for x, y in ((a1, a0), (b1, b0), (a1, b1)):
        assert np.array_equal(np.asarray(x).view(np.uint64), np.asarray(y).view(np.uint64))
