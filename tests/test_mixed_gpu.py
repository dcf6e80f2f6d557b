"""Mixed-precision path (SGNB_MIXED) against the FP64 oracle: configuration 3.

FP32 deviations from the lake at rest with the hydrostatic balance, state, RK accumulation,
error estimate and controller in FP64. Checks: rhs accuracy per field; the lake at rest is
as exact as the FP64 path (the FP32 part vanishes identically at rest); the eta L2 error
after configuration 1's 100 accepted steps (the reference's own step sequence) stays at or
below 1e-6, and L2 and Linf below 1e-6 over 100 steps at a stable fixed step; the lake at
rest over seeded random bathymetry (5 Gaussian bumps) keeps its residual at the FP64
oracle's level over many steps.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
import sgnb
from cases import bump_case, cfg1_case, cfg3_lake_case, lake_case
from conftest import rel_per_field

pytestmark = pytest.mark.gpu

RHS_TOL = 2e-5    # FP32 arithmetic on O(1) terms, relative per field
ETA_TOL = 1e-6    # eta error vs the FP64 oracle (L2 and Linf)


@pytest.mark.parametrize("bc", [0, 1])
def test_mixed_rhs_accuracy(bc):
    kw, U = bump_case(bc, Nx=17, Ny=9)
    R = O.Oracle(**kw).rhs(U)
    with sgnb.SGN2DB200(precision=sgnb.MIXED, **kw) as d:
        Rm = d.rhs(U)
    assert rel_per_field(Rm, R) < RHS_TOL


@pytest.mark.parametrize("bc", [0, 1])
def test_mixed_lake_at_rest(bc):
    kw, _ = bump_case(bc)
    o = O.Oracle(**kw)
    U = lake_case(o.bathymetry()["Hnod"], o.Nd)
    ref = np.abs(o.rhs(U)).max()
    with sgnb.SGN2DB200(precision=sgnb.MIXED, **kw) as d:
        res = np.abs(d.rhs(U)).max()
    assert res < 1e-12 and res <= 10 * max(ref, 1e-16)


def eta_errors(u, ref, Hnod, qw, Nd, J):
    w = np.tile(np.outer(qw, qw).reshape(-1), Nd // 25) * J
    e = (u[:Nd] - Hnod) - (ref[:Nd] - Hnod)
    return np.sqrt(np.sum(w * e * e)), np.abs(e).max()


def _eta_error_fixed_steps(kw, U, dt, n):
    o = O.Oracle(**kw)
    ref = U.copy()
    t = 0.0
    for _ in range(n):
        ref = o.bs3_step(ref, t, dt)
        t += dt
    with sgnb.SGN2DB200(precision=sgnb.MIXED, **kw) as d:
        d.upload(U)
        d.bs3_steps(0.0, np.full(n, dt))
        um = d.download()
    qw = o.tables()["qw"]
    H = o.bathymetry()["Hnod"]
    J = (0.5 * kw["Lx"] / kw["Nx"]) * (0.5 * kw["Ly"] / kw["Ny"])
    return eta_errors(um, ref, H, qw, o.Nd, J)


def test_cfg3_eta_error_stable_steps(golden):
    """Configuration 1's shape and state, 100 BS3 steps at a fixed stable step
    (0.4 x the CFL-0.5 step), the FP64 oracle taking the same steps: eta L2 and Linf
    errors of the mixed path below 1e-6 (measured ~1e-10)."""
    kw, U = cfg1_case()
    dt = 0.4 * float(golden["cfg1_dt0"][0])
    l2, linf = _eta_error_fixed_steps(kw, U, dt, 100)
    print(f"stable-step eta error: L2 {l2:.3e} Linf {linf:.3e}")
    assert l2 < ETA_TOL and linf < ETA_TOL, (l2, linf)


def test_cfg3_eta_error_reference_steps(golden):
    """Configuration 3 as written: configuration 1's shape and state, the reference's own
    100 accepted adaptive steps (tests/golden: cfg1_dts, from src/solver/rk.cpp:67-164), the
    FP64 oracle taking the same steps: eta L2 (quadrature-weighted over the domain) at
    most 1e-6 after the 100 steps. The sequence runs near the edge of linear stability,
    so grid-scale noise grows by orders of magnitude (the FP64 fast path, whose rounding
    differs from the CPU's only in the last bit, ends ~1e-11 away); FP32 storage of k alone
    would end near 1e-7 (tests/test_mixed_bounds.py)."""
    kw, U = cfg1_case()
    o = O.Oracle(**kw)
    dts = golden["cfg1_dts"]
    assert dts.size == 100
    ref = U.copy()
    t = 0.0
    for dt in dts:
        ref = o.bs3_step(ref, t, dt)
        t += dt
    qw = o.tables()["qw"]
    H = o.bathymetry()["Hnod"]
    J = (0.5 * kw["Lx"] / kw["Nx"]) * (0.5 * kw["Ly"] / kw["Ny"])
    err = {}
    for prec in (sgnb.FP64_FAST, sgnb.MIXED):
        with sgnb.SGN2DB200(precision=prec, **kw) as d:
            d.upload(U)
            d.bs3_steps(0.0, dts)
            err[prec] = eta_errors(d.download(), ref, H, qw, o.Nd, J)
    print("eta L2 / Linf after the reference's 100 steps: fast %.2e / %.2e, mixed %.2e / %.2e"
          % (*err[sgnb.FP64_FAST], *err[sgnb.MIXED]))
    assert err[sgnb.FP64_FAST][0] < 1e-9
    assert err[sgnb.MIXED][0] <= ETA_TOL


def test_cfg3_lake_at_rest_random_bathymetry():
    """Seeded 5-bump bathymetry in a walled basin (the bumps are not periodic), lake at
    rest: the residual of the mixed path is at the FP64 oracle's level, and 50 steps at
    the CFL step (dtMax caps the controller, which would otherwise grow dt fivefold per
    step on a zero error estimate) keep the lake at rest like the FP64 path."""
    kw = dict(cfg3_lake_case(), bc_x=1, bc_y=1)
    o = O.Oracle(**kw)
    H = o.bathymetry()["Hnod"]
    U = lake_case(H, o.Nd)
    r64 = np.abs(o.rhs(U)).max()
    dtc = 0.5 * (20.0 / 128) / 9 / np.sqrt(9.81 * 1.0 + kw["c"] ** 2)
    opt = sgnb.AdaptiveRKOptions(dtMax=dtc)
    drift, res = {}, {}
    for prec in (sgnb.FP64_FAST, sgnb.MIXED):
        with sgnb.SGN2DB200(precision=prec, **kw) as d:
            res[prec] = np.abs(d.rhs(U)).max()
            d.upload(U)
            st = d.integrate_steps(0.0, dtc, 50, opt)
            u = d.download()
        assert st.accepted == 50
        drift[prec] = max(np.abs(u[: o.Nd] - H).max(), np.abs(u[o.Nd:]).max())
    print("rest residual", r64, res, "drift after 50 steps:", drift)
    assert res[sgnb.MIXED] <= max(10 * r64, 1e-13)
    assert drift[sgnb.MIXED] < 1e-12
    assert drift[sgnb.MIXED] <= 10 * max(drift[sgnb.FP64_FAST], 1e-15)
