"""Forty seeded random cases through the device right-hand side.

tests/cases.py random_case: meshes of 2..9 x 2..9 elements, each direction periodic or
walled, random g, gamma, c and Manning coefficient, GLL or Gauss-Legendre points, flat,
constant or Gaussian-bump bathymetry, a smooth random state. The oracle's rhs of the same
cases is pinned to the reference's bit for bit (tests/test_oracle.py). Bars:
* exact mode: bit for bit; with Manning friction to the last-bit rounding of the cube root
  (1e-15 relative per field: the device's and the host's cbrt may round differently);
* fast mode: 1e-13 relative per field (GLL), 2e-13 (Gauss-Legendre points, whose traces
  combine five nodes);
* mixed mode (GLL only): its FP32 bar, 2e-5;
* frozen step sequences on the first twelve cases without friction: three bs3Step and
  three rk4Step steps, exact mode bit for bit.
"""
from __future__ import annotations

import pytest

import oracle as O
import sgnb
from cases import random_case
from conftest import bits_equal, rel_per_field

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", range(40))
def test_random_case_rhs(seed):
    kw, U = random_case(seed)
    R = O.Oracle(**kw).rhs(U)
    gauss = kw["points"] == O.POINTS_GAUSS
    with sgnb.SGN2DB200(precision=sgnb.FP64_EXACT, **kw) as d:
        if kw["nManning"] > 0.0:
            assert rel_per_field(d.rhs(U), R) < 1e-15
        else:
            assert bits_equal(d.rhs(U), R)
    with sgnb.SGN2DB200(precision=sgnb.FP64_FAST, **kw) as d:
        assert rel_per_field(d.rhs(U), R) < (2e-13 if gauss else 1e-13)
    if not gauss:
        with sgnb.SGN2DB200(precision=sgnb.MIXED, **kw) as d:
            assert rel_per_field(d.rhs(U), R) < 2e-5


@pytest.mark.parametrize("seed", range(12))
def test_random_case_fixed_steps(seed):
    kw, U = random_case(seed)
    if kw["nManning"] > 0.0:
        kw = dict(kw, nManning=0.0)  # bit for bit needs the same cube roots
    o = O.Oracle(**kw)
    dt = 0.5 * o.cfl_time_step(U, 0.5)
    dts = [dt, 0.9 * dt, 1.1 * dt]
    ref3, ref4 = U.copy(), U.copy()
    t = 0.0
    for h in dts:
        ref3 = o.bs3_step(ref3, t, h)
        ref4 = o.rk4_step(ref4, t, h)
        t += h
    with sgnb.SGN2DB200(precision=sgnb.FP64_EXACT, **kw) as d:
        d.upload(U)
        d.bs3_steps(0.0, dts)
        assert bits_equal(d.download(), ref3)
        d.upload(U)
        d.rk4_steps(0.0, dts)
        assert bits_equal(d.download(), ref4)
