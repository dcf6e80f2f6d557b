"""What FP32 arithmetic can and cannot do on configuration 3's accuracy bar (CPU, the oracle).

Configuration 3 asks for an eta error of at most 1e-6 (quadrature-weighted L2 over the
domain) against the FP64 oracle after configuration 1's 100 accepted adaptive steps (the
reference's own step sequence, tests/golden: cfg1_dts). That sequence runs near the edge of
linear stability for grid-scale modes (src/solver/rk.cpp:112-161), so white noise grows by
orders of magnitude (test_oracle.py::test_cfg1_controller_sensitivity). Whether the bar can
be met in FP32 then depends on where the rounding enters. These tests replay the sequence
with the oracle's right-hand side and BS3(2) combinations (src/solver/rk.cpp:41-54, the same
operation order: the unmodified replay is bit-identical to the oracle's bs3Step) while
rounding chosen quantities to FP32:

* every stage derivative k stored in FP32 (what the mixed mode's k buffers do): the error
  peaks near step 10 and decays to about 1e-7, under the bar;
* the discharges hw and hp of every stage input rounded to FP32 as well: still about 1e-7;
* the discharges hu and hv of every stage input rounded to FP32: about 4e-6, over the bar.
  Their 5-point derivative (the mass flux) turns per-node rounding into grid-scale noise
  in dh/dt, which the sequence amplifies.

So the mixed mode keeps hu, hv and the terms linear in them in FP64
(csrc/sgnb_kernels_mixed.cuh); tests/test_mixed_gpu.py holds the device to the bar.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from cases import cfg1_case

ETA_TOL = 1e-6


def _f32(a):
    return a.astype(np.float32).astype(np.float64)


@pytest.fixture(scope="module")
def cfg1_run(golden):
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
    J = (0.5 * kw["Lx"] / kw["Nx"]) * (0.5 * kw["Ly"] / kw["Ny"])
    w = np.tile(np.outer(qw, qw).reshape(-1), o.Nd // 25) * J
    return o, U, dts, ref, w


def _replay(o, U, dts, round_inputs=(), round_k=False):
    """bs3Step replay with FP32 rounding of the listed stage-input fields and/or of k."""
    Nd = o.Nd

    def f(y):
        y = y.copy()
        for v in round_inputs:
            y[v * Nd:(v + 1) * Nd] = _f32(y[v * Nd:(v + 1) * Nd])
        k = o.rhs(y)
        return _f32(k) if round_k else k

    u = U.copy()
    for dt in dts:
        k1 = f(u)
        k2 = f(u + (0.5 * dt) * k1)
        k3 = f(u + (0.75 * dt) * k2)
        u = u + dt * ((2.0 / 9.0) * k1 + (1.0 / 3.0) * k2 + (4.0 / 9.0) * k3)
    return u


def _eta_l2(u, ref, w, Nd):
    e = u[:Nd] - ref[:Nd]  # eta differences are h differences (same still depth)
    return float(np.sqrt(np.sum(w * e * e)))


def test_replay_is_the_oracle_step(cfg1_run):
    o, U, dts, ref, w = cfg1_run
    assert np.array_equal(_replay(o, U, dts[:3]).view(np.uint64),
                          o.bs3_step(o.bs3_step(o.bs3_step(U, 0.0, dts[0]), dts[0], dts[1]),
                                     dts[0] + dts[1], dts[2]).view(np.uint64))


def test_fp32_k_and_hw_hp_stay_under_the_bar(cfg1_run):
    o, U, dts, ref, w = cfg1_run
    e_k = _eta_l2(_replay(o, U, dts, round_k=True), ref, w, o.Nd)
    e_whp = _eta_l2(_replay(o, U, dts, round_inputs=(3, 4), round_k=True), ref, w, o.Nd)
    print(f"eta L2 after 100 steps: k in FP32 {e_k:.2e}; k, hw, hp in FP32 {e_whp:.2e}")
    assert 0 < e_k < 0.3 * ETA_TOL
    assert 0 < e_whp < 0.3 * ETA_TOL


def test_fp32_hu_hv_inputs_break_the_bar(cfg1_run):
    o, U, dts, ref, w = cfg1_run
    e = _eta_l2(_replay(o, U, dts, round_inputs=(1, 2), round_k=True), ref, w, o.Nd)
    print(f"eta L2 after 100 steps: k, hu, hv in FP32 {e:.2e}")
    assert e > 2 * ETA_TOL
