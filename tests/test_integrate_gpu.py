"""The device-resident Bogacki-Shampine 3(2) loop against the CPU oracle.

* frozen-dt replay (consecutive bs3Step, src/solver/rk.cpp:41-54) is bit-identical in the
  exact mode;
* free adaptive runs take the same accept/reject sequence as the reference and end within
  1e-10 relative (the reference's own GPU gate is 1e-6, test/test_cuda_sgn2d.cu:96-128);
  the error norm is reduced in a different order than the CPU's sequential sum, so the
  controller's dt differs in the last bits;
* mass is conserved to 1e-13; a NaN state stops the run with SGNB_ERR_NAN instead of
  looping forever; dtMin aborts like the reference (stats.aborted, state at the last
  accepted step).
"""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

import oracle as O
import sgnb
from cases import bump_case, cfg1_case, CFG1_STEPS
from conftest import bits_equal, rel_per_field

pytestmark = pytest.mark.gpu


def accepted_dts(o, U, tEnd, dt0, **opts):
    _, _, log = o.integrate_adaptive(U, 0.0, tEnd, dt0, max_log=100000, **opts)
    return log[log[:, 3] == 1][:, 1].copy()


@pytest.mark.parametrize("bc", [0, 1])
def test_frozen_replay_bitwise(bc):
    kw, U = bump_case(bc)
    o = O.Oracle(**kw)
    dt0 = o.cfl_time_step(U, 0.5)
    dts = accepted_dts(o, U, 30 * dt0, dt0)[:25]
    ref = U.copy()
    t = 0.0
    for dt in dts:
        ref = o.bs3_step(ref, t, dt)
        t += dt
    with sgnb.SGN2DB200(precision=sgnb.FP64_EXACT, **kw) as d:
        d.upload(U)
        d.bs3_steps(0.0, dts)
        assert bits_equal(d.download(), ref)
    with sgnb.SGN2DB200(precision=sgnb.FP64_FAST, **kw) as d:
        d.upload(U)
        d.bs3_steps(0.0, dts)
        assert rel_per_field(d.download(), ref) < 1e-12


@pytest.mark.parametrize("prec", [sgnb.FP64_EXACT, sgnb.FP64_FAST])
def test_adaptive_matches_reference_run(golden, prec):
    """The reference's GPU gate run (tEnd 0.3, atol 1e-10, rtol 1e-8) and the committed
    golden short run (tEnd 0.05)."""
    kw, U = bump_case()
    o = O.Oracle(**kw)
    dt0 = o.cfl_time_step(U, 0.5)
    opt = sgnb.AdaptiveRKOptions(atol=1e-10, rtol=1e-8)
    for tEnd in (0.05, 0.3):
        uo, so, _ = o.integrate_adaptive(U, 0.0, tEnd, dt0, atol=1e-10, rtol=1e-8)
        with sgnb.SGN2DB200(precision=prec, **kw) as d:
            d.upload(U)
            M0 = d.mass()
            st = d.integrate_adaptive(0.0, tEnd, dt0, opt)
            ug = d.download()
            M1 = d.mass()
        assert (st.accepted, st.rejected, st.rhsEvals) == (so["accepted"], so["rejected"],
                                                           so["rhsEvals"])
        assert st.tReached == so["tReached"] and st.aborted == 0
        assert rel_per_field(ug, uo) < 1e-10
        assert abs(M1 - M0) / abs(M0) < 1e-13
        if tEnd == 0.05:
            assert list(golden["run_stats"]) == [st.accepted, st.rejected, st.rhsEvals]
            assert rel_per_field(ug, golden["run_U"]) < 1e-10


def test_cfg1_frozen_replay_bitwise(golden):
    """Configuration 1, the reference's 100 accepted steps replayed with their step sizes:
    the final state is the reference's integrateAdaptive result bit for bit (bs3Step and
    the FSAL loop take identical steps, src/solver/rk.h:44-50)."""
    kw, U = cfg1_case()
    dts = golden["cfg1_dts"]
    assert dts.size == CFG1_STEPS and float(np.sum(dts)) > 0
    with sgnb.SGN2DB200(precision=sgnb.FP64_EXACT, **kw) as d:
        d.upload(U)
        d.bs3_steps(0.0, dts)
        u = d.download()
    assert hashlib.sha256(u.tobytes()).hexdigest() == str(golden["cfg1_final_sha"][0])


@pytest.mark.parametrize("prec", [sgnb.FP64_EXACT, sgnb.FP64_FAST])
def test_cfg1_hundred_steps(golden, prec):
    """Configuration 1, free adaptive run to the time of the reference's 100th accepted step.

    On this configuration the reference's own controller amplifies round-off: a 1-ulp change
    of dt0 grows to ~1e-4 relative in the error norm within 9 steps
    (test_oracle.py::test_cfg1_controller_sensitivity). The device reduces the error norm
    in another order than the CPU's sequential sum, so its dt sequence drifts from the
    reference's at that level, and tEnd (exactly the reference's t_100) may be reached with
    one extra, tiny step. The states agree within the reference's own GPU gate of 1e-6
    (test/test_cuda_sgn2d.cu:124)."""
    kw, U = cfg1_case()
    dt0 = float(golden["cfg1_dt0"][0])
    tEnd = float(golden["cfg1_tEnd"][0])
    idx = golden["cfg1_idx"]
    with sgnb.SGN2DB200(precision=prec, **kw) as d:
        d.upload(U)
        assert d.cfl_time_step(0.5) == dt0
        st = d.integrate_adaptive(0.0, tEnd, dt0)
        u = d.download()
    ref_stats = list(golden["cfg1_stats"])
    assert st.accepted in (CFG1_STEPS, CFG1_STEPS + 1) and st.rejected == ref_stats[1]
    assert st.tReached == pytest.approx(tEnd, abs=1e-15)
    ref = golden["cfg1_final_samples"]
    assert np.abs(u[idx] - ref).max() <= 1e-6 * np.abs(ref).max()


def test_nan_state_stops_with_status():
    kw, U = bump_case()
    U = U.copy()
    U[137] = np.nan
    with sgnb.SGN2DB200(precision=sgnb.FP64_EXACT, **kw) as d:
        d.upload(U)
        with pytest.raises(sgnb.SgnbError) as ei:
            d.integrate_adaptive(0.0, 0.1, 1e-3)
        assert ei.value.status == 4
        st = d.integrate_adaptive(0.0, 0.1, 1e-3, raise_on_nan=False)
        assert st.aborted == 2 and st.accepted == 0


def test_dtmin_abort_keeps_last_accepted_state():
    kw, U = bump_case()
    o = O.Oracle(**kw)
    dt0 = o.cfl_time_step(U, 0.5)
    opts = dict(atol=1e-14, rtol=1e-14, dtMin=1e-4)
    uo, so, _ = o.integrate_adaptive(U, 0.0, 0.1, dt0, **opts)
    assert so["aborted"] == 1
    with sgnb.SGN2DB200(precision=sgnb.FP64_EXACT, **kw) as d:
        d.upload(U)
        st = d.integrate_adaptive(0.0, 0.1, dt0, sgnb.AdaptiveRKOptions(**opts))
        ug = d.download()
    assert st.aborted == 1
    assert (st.accepted, st.rejected) == (so["accepted"], so["rejected"])
    assert rel_per_field(ug, uo) < 1e-10


def test_zero_length_interval():
    kw, U = bump_case()
    with sgnb.SGN2DB200(precision=sgnb.FP64_EXACT, **kw) as d:
        d.upload(U)
        st = d.integrate_adaptive(0.5, 0.5, 1e-3)
        assert (st.accepted, st.rejected, st.rhsEvals) == (0, 0, 1)
        assert bits_equal(d.download(), U)


def test_device_loop_matches_host_loop_and_relaunches(monkeypatch):
    """The device-side loop (a CUDA-graph WHILE node whose controller sets the condition)
    and the host-launched loop (SGNB_HOST_LOOP=1) run the same kernels: bit for bit the
    same run. 5000 steps cross the device loop's 4096-attempt bound on one graph launch,
    so the host relaunches it once; launch counts are exact on the device loop."""
    kw, U = bump_case(1, Nx=4, Ny=3, Lx=5.0, Ly=4.0)
    runs = {}
    for mode in ("device", "host"):
        if mode == "host":
            monkeypatch.setenv("SGNB_HOST_LOOP", "1")
        else:
            monkeypatch.delenv("SGNB_HOST_LOOP", raising=False)
        with sgnb.SGN2DB200(precision=sgnb.FP64_EXACT, **kw) as d:
            d.upload(U)
            dt0 = d.cfl_time_step(0.5)
            st = d.integrate_steps(0.0, dt0, 5000)
            runs[mode] = (d.download(), st)
    (ud, sd), (uh, sh) = runs["device"], runs["host"]
    assert (sd.accepted, sd.rejected, sd.attempts) == (sh.accepted, sh.rejected, sh.attempts)
    assert sd.accepted == 5000 and sd.attempts > 4096
    assert bits_equal(ud, uh) and sd.tReached == sh.tReached
    assert sd.kernel_launches == 1 + 4 * sd.attempts
    assert sh.kernel_launches >= sd.kernel_launches
