"""The fast arithmetic mode's own reciprocal and square root (Newton-Raphson from the
hardware estimates) against the IEEE results of the same device, in ulps.

fast_rcp serves 1/h in the primitive variables and 1/sc in the scaled embedded error;
fast_sqrt serves the wave speed sqrt(max(g h + p + c^2, 0)) of the Rusanov flux. Both are
held to 2 ulp over normal arguments from 1e-300 to 1e300; the square root hands zero,
subnormal, infinite, negative and NaN arguments to the IEEE square root unchanged.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import sgnb

pytestmark = pytest.mark.gpu


def fast_math(fn, x):
    import torch

    xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).cuda()
    yd = torch.empty_like(xd)
    torch.cuda.synchronize()
    rc = sgnb.lib().sgnb_fast_math(fn, C.cast(C.c_void_p(xd.data_ptr()), sgnb._dp),
                                   C.cast(C.c_void_p(yd.data_ptr()), sgnb._dp), xd.numel(),
                                   None)
    assert rc == 0
    return xd, yd


def ulps(a, b):
    return np.abs(a - b) / np.spacing(np.abs(b))


def arguments(seed=5):
    rng = np.random.default_rng(seed)
    x = 10.0 ** rng.uniform(-300, 300, 1 << 20)
    dmin = np.finfo(np.float64).tiny
    special = [dmin, np.nextafter(dmin, 1.0), 1.0, 2.0, 4.0, 0.5, np.nextafter(1.0, 0.0),
               np.nextafter(1.0, 2.0), 9.81, 0.45, 1e-8, 3.0 * np.sqrt(9.81)]
    depths = rng.uniform(1e-3, 1e2, 1 << 16)  # depths, wave-speed arguments, error scales
    return np.concatenate([x, special, depths])


def test_fast_reciprocal_within_two_ulp():
    x = arguments()
    xd, yd = fast_math(0, x)
    ref = (1.0 / xd).cpu().numpy()
    err = ulps(yd.cpu().numpy(), ref)
    assert err.max() <= 2.0, (err.max(), x[err.argmax()])
    neg = -x[:1000]
    _, yn = fast_math(0, neg)
    assert ulps(yn.cpu().numpy(), 1.0 / neg).max() <= 2.0


def test_fast_sqrt_within_two_ulp_and_ieee_edges():
    import torch

    x = arguments(7)
    xd, yd = fast_math(1, x)
    err = ulps(yd.cpu().numpy(), torch.sqrt(xd).cpu().numpy())
    assert err.max() <= 2.0, (err.max(), x[err.argmax()])
    edges = np.array([0.0, -0.0, 5e-324, 1e-310, np.inf, -1.0, np.nan,
                      np.finfo(np.float64).max])
    ed, ye = fast_math(1, edges)
    want = torch.sqrt(ed).cpu().numpy()
    got = ye.cpu().numpy()
    assert np.array_equal(np.isnan(got), np.isnan(want))
    fin = ~np.isnan(want)
    assert np.array_equal(got[fin].view(np.uint64), want[fin].view(np.uint64))
