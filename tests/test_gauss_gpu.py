"""Gauss-Legendre solution points (PointSet::GaussLegendre) on the device.

The reference admits them on a flat bottom only (H = 0, src/solver/sgn2d.cpp:46-47). Their
face traces are interpolated with lL / lR (sgn2d.cpp:141-177) instead of being the edge
nodes: a trace pre-pass stores every element's four face traces, and the fused kernels'
GAUSS variant reads its neighbours' traces from it and forms its own. Checked here:

* the right-hand side, exact mode: bit for bit the oracle's (pinned to the reference's
  Gauss-point solver) and the committed golden rhs; periodic, walls, partial tiles,
  Manning friction (to the last-bit rounding of cbrt); fast mode within 2e-13 relative per field (FAST_TOL: each trace
  combines five nodes with sum |lL| = 3.3, against one node for GLL points, so the fast
  mode's FMA contractions and reciprocals meet about three times the rounding);
* BS3(2) frozen replay bit for bit, adaptive runs with the oracle's accepted / rejected
  counts and the golden short run;
* mass and energy with the Gauss quadrature weights.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
import sgnb
from cases import gauss_case
from conftest import bits_equal, rel_per_field

pytestmark = pytest.mark.gpu


FAST_TOL = 2e-13


def oracle_of(kw):
    return O.Oracle(**kw)


def device_of(kw, prec):
    return sgnb.SGN2DB200(precision=prec, **kw)


@pytest.mark.parametrize("bc", [0, 1])
@pytest.mark.parametrize("Nx,Ny", [(8, 6), (11, 5), (9, 13), (2, 2)])
def test_rhs_exact_bitwise_and_fast(bc, Nx, Ny):
    kw, U = gauss_case(bc, Nx=Nx, Ny=Ny, Lx=1.25 * Nx, Ly=1.3 * Ny)
    R = oracle_of(kw).rhs(U)
    with device_of(kw, sgnb.FP64_EXACT) as d:
        assert bits_equal(d.rhs(U), R)
    with device_of(kw, sgnb.FP64_FAST) as d:
        assert rel_per_field(d.rhs(U), R) < FAST_TOL


def test_rhs_golden_and_manning(golden):
    kw, U = gauss_case()
    with device_of(kw, sgnb.FP64_EXACT) as d:
        assert bits_equal(d.rhs(U), golden["gauss_R"])
    kwm = dict(kw, nManning=0.03)
    R = oracle_of(kwm).rhs(U)
    assert not bits_equal(R, golden["gauss_R"])
    with device_of(kwm, sgnb.FP64_EXACT) as d:
        # the device's and the host's cube roots may round differently in the last bit
        assert rel_per_field(d.rhs(U), R) < 1e-15


def test_tables_and_quadrature():
    kw, U = gauss_case(0, Nx=6, Ny=4, Lx=6.0, Ly=4.0)
    o = oracle_of(kw)
    with device_of(kw, sgnb.FP64_EXACT) as d:
        x, y = d.node_coords()
        xo, yo = o.node_coords()
        assert bits_equal(x, xo) and bits_equal(y, yo)
        d.upload(U)
        assert abs(d.mass() - o.mass(U)) <= 1e-14 * abs(o.mass(U))
        assert abs(d.energy() - o.energy(U)) <= 1e-13 * abs(o.energy(U))
        assert abs(d.max_wave_speed() - o.max_wave_speed(U)) <= 1e-15 * o.max_wave_speed(U)


@pytest.mark.parametrize("bc", [0, 1])
def test_frozen_replay_bitwise(bc):
    kw, U = gauss_case(bc)
    o = oracle_of(kw)
    dt0 = o.cfl_time_step(U, 0.5)
    _, _, log = o.integrate_adaptive(U, 0.0, 30 * dt0, dt0, max_log=100000)
    dts = log[log[:, 3] == 1][:20, 1].copy()
    ref = U.copy()
    t = 0.0
    for dt in dts:
        ref = o.bs3_step(ref, t, dt)
        t += dt
    with device_of(kw, sgnb.FP64_EXACT) as d:
        d.upload(U)
        d.bs3_steps(0.0, dts)
        assert bits_equal(d.download(), ref)
    with device_of(kw, sgnb.FP64_FAST) as d:
        d.upload(U)
        d.bs3_steps(0.0, dts)
        assert rel_per_field(d.download(), ref) < 1e-12


@pytest.mark.parametrize("prec", [sgnb.FP64_EXACT, sgnb.FP64_FAST])
def test_adaptive_matches_reference_run(golden, prec):
    kw, U = gauss_case()
    o = oracle_of(kw)
    dt0 = o.cfl_time_step(U, 0.5)
    uo, so, _ = o.integrate_adaptive(U, 0.0, 0.05, dt0, atol=1e-10, rtol=1e-8)
    assert [so["accepted"], so["rejected"], so["rhsEvals"]] == list(golden["gauss_run_stats"])
    with device_of(kw, prec) as d:
        d.upload(U)
        M0 = d.mass()
        st = d.integrate_adaptive(0.0, 0.05, dt0, sgnb.AdaptiveRKOptions(atol=1e-10, rtol=1e-8))
        ug = d.download()
        assert abs(d.mass() - M0) <= 1e-13 * abs(M0)
    assert [st.accepted, st.rejected, st.rhsEvals] == list(golden["gauss_run_stats"])
    assert st.tReached == so["tReached"]
    assert rel_per_field(ug, golden["gauss_run_U"]) < 1e-10
    # two kernels per right-hand side: the trace pre-pass and the fused kernel
    assert st.kernel_launches >= 2 + 7 * (st.accepted + st.rejected)


def test_gauss_refused_where_not_built():
    kw, U = gauss_case(0)
    with device_of(kw, sgnb.FP64_FAST) as d:
        from sgnb.adjoint import SGNAdjoint

        with pytest.raises(sgnb.SgnbError) as ei:
            SGNAdjoint(d, [1e-3], [0])
        assert ei.value.status == 2
    with pytest.raises(sgnb.SgnbError) as ei:
        sgnb.SGNBatch([dict(kw)])
    assert ei.value.status == 2
