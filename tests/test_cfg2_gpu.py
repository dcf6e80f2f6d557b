"""Configuration 2 at full size (2048 x 1024 elements, 262,144,000 DOF) against the CPU oracle.

The benchmark's own inputs: reflective walls on the 40 x 20 basin, the elliptic shoal on the
0.45 plane (BATHY_SHOAL) and the 8 seeded random-phase sines, built by the same generator the
benchmark uses (sgnb.workloads.cfg2_state_torch). The oracle (oracle/sgn_oracle.c) is pinned
bit for bit to the reference's CPU solver on the same generator through mirror doubling
(tests/test_oracle.py::test_cfg2_generator_vs_reference), so these are the reference's GPU
gates (test/test_cuda_sgn2d.cu:66-80: GPU rhs == CPU rhs) on the benchmarked configuration:

* exact mode: the right-hand side bit for bit (src/solver/sgn2d.cpp:125-290);
* fast mode: within 2e-13 relative per field. The fast mode contracts the 5-point
  derivatives in another order (FMA, lift first, one multiplication by 1/J), so it differs
  from the CPU by the round-off of those sums. For the momentum fields that round-off is
  relative to the hydrostatic flux 0.5 g (h^2 - H^2) ~ 0.09 rather than to its derivative:
  the derivative cancels about a hundredfold inside an element and is then divided by
  J = 0.0098 at this element size (measured 6.5e-14 absolute, 1.2e-13 of the largest value;
  the reference's own GPU gate is 1e-12, test/test_cuda_sgn2d.cu:66-80);
* exact mode: two frozen BS3(2) steps (bs3Step, src/solver/rk.cpp:41-54) bit for bit.

Each oracle right-hand side of the full state takes about 5 s on one host core.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
import sgnb
from conftest import bits_equal, rel_per_field
from sgnb import workloads as W

pytestmark = pytest.mark.gpu

FAST_TOL = 2e-13  # at configuration 2's element size, see above


@pytest.fixture(scope="module")
def cfg2():
    kw = W.cfg2_solver_args()
    U = W.cfg2_state_torch(device="cuda").cpu().numpy()
    return kw, U, O.Oracle(**kw)


def test_cfg2_full_size_rhs(cfg2):
    kw, U, ref = cfg2
    assert U.size == 5 * 25 * 2048 * 1024
    R = ref.rhs(U)
    assert np.isfinite(R).all()
    with sgnb.SGN2DB200(precision=sgnb.FP64_EXACT, **kw) as d:
        Rg = d.rhs(U)
        assert bits_equal(Rg, R), f"max |diff| {np.abs(Rg - R).max():.3e}"
    del Rg
    with sgnb.SGN2DB200(precision=sgnb.FP64_FAST, **kw) as d:
        Rf = d.rhs(U)
        for v in range(5):
            a, b = Rf[v * ref.Nd:(v + 1) * ref.Nd], R[v * ref.Nd:(v + 1) * ref.Nd]
            i = int(np.argmax(np.abs(a - b)))
            print(f"field {v}: max|R| {np.abs(b).max():.3e} max|diff| {np.abs(a - b)[i]:.3e} "
                  f"at node {i} (R {b[i]:.3e})")
        assert rel_per_field(Rf, R) < FAST_TOL
        # the step size of the same state
        d.upload(U)
        assert d.cfl_time_step(0.5) == ref.cfl_time_step(U, 0.5)


def test_cfg2_full_size_two_frozen_steps(cfg2):
    kw, U, ref = cfg2
    dt0 = ref.cfl_time_step(U, 0.5)
    dts = [dt0, 0.9 * dt0]
    u = U
    t = 0.0
    for dt in dts:
        u = ref.bs3_step(u, t, dt)
        t += dt
    with sgnb.SGN2DB200(precision=sgnb.FP64_EXACT, **kw) as d:
        d.upload(U)
        d.bs3_steps(0.0, dts)
        ug = d.download()
    assert bits_equal(ug, u), f"max |diff| {np.abs(ug - u).max():.3e}"
    assert not bits_equal(u, U)
