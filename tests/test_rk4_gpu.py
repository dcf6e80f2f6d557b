"""Classical RK4 steps (rk4Step, src/solver/rk.cpp:23-38) on the device.

sgnb_rk4_steps evaluates R(u), then the fused stage kernel with the stage coefficients 1/2,
1/2 and 1, then the update u += dt/6 (k1 + 2 k2 + 2 k3 + k4). Checked against the
oracle's rk4_step, which is pinned bit for bit to the reference's rk4Step:
* exact mode bit for bit over several steps: periodic and walls, partial tiles, Manning
  friction, Gauss-Legendre points;
* fast mode within 1e-12 relative per field;
* fourth-order convergence of the step against a reference solution with steps 1/4 as long;
* an empty list leaves the state alone; the mixed mode refuses (FP64 modes only).
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
import sgnb
from cases import bump_case, gauss_case
from conftest import bits_equal, rel_per_field

pytestmark = pytest.mark.gpu


def oracle_rk4(o, U, dts):
    u = U.copy()
    t = 0.0
    for dt in dts:
        u = o.rk4_step(u, t, dt)
        t += dt
    return u


def device_rk4(kw, prec, U, dts):
    with sgnb.SGN2DB200(precision=prec, **kw) as d:
        d.upload(U)
        d.rk4_steps(0.0, dts)
        return d.download()


@pytest.mark.parametrize("bc", [0, 1])
@pytest.mark.parametrize("Nx,Ny", [(8, 6), (11, 5), (2, 2)])
def test_rk4_bitwise_exact_and_fast(bc, Nx, Ny):
    kw, U = bump_case(bc, Nx=Nx, Ny=Ny, Lx=1.25 * Nx, Ly=1.3 * Ny)
    o = O.Oracle(**kw)
    dt = o.cfl_time_step(U, 0.5)
    dts = [dt, 0.7 * dt, 1.1 * dt, dt]
    ref = oracle_rk4(o, U, dts)
    assert bits_equal(device_rk4(kw, sgnb.FP64_EXACT, U, dts), ref)
    assert rel_per_field(device_rk4(kw, sgnb.FP64_FAST, U, dts), ref) < 1e-12


def test_rk4_manning_and_gauss_points():
    kw, U = bump_case(1, Nx=9, Ny=7, Lx=11.0, Ly=8.0)
    kw = dict(kw, nManning=0.03)
    o = O.Oracle(**kw)
    dt = o.cfl_time_step(U, 0.5)
    ref = oracle_rk4(o, U, [dt, dt])
    # the device's and the host's cube roots may round differently in the last bit
    assert rel_per_field(device_rk4(kw, sgnb.FP64_EXACT, U, [dt, dt]), ref) < 1e-14
    for bc in (0, 1):
        kwg, Ug = gauss_case(bc, Nx=9, Ny=5, Lx=11.0, Ly=6.0)
        og = O.Oracle(**kwg)
        dtg = og.cfl_time_step(Ug, 0.5)
        refg = oracle_rk4(og, Ug, [dtg, 0.5 * dtg, dtg])
        assert bits_equal(device_rk4(kwg, sgnb.FP64_EXACT, Ug, [dtg, 0.5 * dtg, dtg]), refg)
        assert rel_per_field(device_rk4(kwg, sgnb.FP64_FAST, Ug, [dtg, 0.5 * dtg, dtg]), refg) < 1e-12


def test_rk4_fourth_order():
    """Halving the step divides the error at a fixed end time by about 2^4 (rk.h:22 names
    rk4Step the convergence-test integrator)."""
    kw, U = bump_case(0, Nx=8, Ny=6)
    with sgnb.SGN2DB200(precision=sgnb.FP64_EXACT, **kw) as d:
        d.upload(U)
        dt0 = d.cfl_time_step(0.4)
    T = 4 * dt0  # the coarse run's steps are the CFL-0.4 step

    def run(m):
        return device_rk4(kw, sgnb.FP64_EXACT, U, [T / m] * m)

    fine = run(64)
    e1 = np.abs(run(4) - fine).max()
    e2 = np.abs(run(8) - fine).max()
    assert 10.0 < e1 / e2 < 24.0


def test_rk4_empty_list_and_mixed_refused():
    kw, U = bump_case(0)
    with sgnb.SGN2DB200(precision=sgnb.FP64_FAST, **kw) as d:
        d.upload(U)
        d.rk4_steps(0.0, [])
        assert bits_equal(d.download(), U)
    with sgnb.SGN2DB200(precision=sgnb.MIXED, **kw) as d:
        d.upload(U)
        with pytest.raises(sgnb.SgnbError) as ei:
            d.rk4_steps(0.0, [1e-3])
        assert ei.value.status == 2
