"""The batched sweep: many uneven instances in one persistent launch per RK stage.

Every instance of a batch must follow the same trajectory as the same instance run alone
through the single-instance device loop (which the other GPU tests pin to the oracle), and
one small instance is also checked against the oracle directly:

* every tile shape and grid: the same accepted / rejected counts as single runs and
  states within 1e-10 relative per field (the batched kernels read each instance's
  constants from shared memory, so FMA contraction may round differently from the
  single-instance kernel in the last bit, and with 16x2 or 4x8 tiles the error partials
  are summed over other tiles);
* the autotuner leaves every instance's state untouched; instances that finish early are
  not advanced by the rest of the batch's attempts; a non-finite instance stops with
  SGNB_ERR_NAN while its neighbours finish normally.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
import sgnb
from cases import G, GAMMA, ALPHA, gll5, make_state, node_coords
from conftest import bits_equal, rel_per_field

pytestmark = pytest.mark.gpu

# uneven sizes: partial tiles in every shape, a one-tile instance, periodic and walls
SIZES = [(10, 6, 1), (17, 9, 0), (33, 5, 1), (8, 4, 1), (24, 13, 0), (5, 31, 1), (48, 20, 1)]


def small_batch(seed=7):
    rng = np.random.default_rng(seed)
    out = []
    for Nx, Ny, bc in SIZES:
        Lx, Ly = 0.25 * Nx, 0.3 * Ny
        H0, crest = 1.0, float(rng.uniform(0.3, 0.9))
        shoal = (H0, crest, 0.55 * Lx, 0.5 * Ly, 0.3 * Lx, 0.25 * Ly)
        kw = dict(P=4, Nx=Nx, Ny=Ny, Lx=Lx, Ly=Ly, g=G, gamma=GAMMA,
                  c=float(rng.uniform(1.5, 6.0)) * np.sqrt(G * H0), bc_x=bc, bc_y=bc,
                  bathy_kind=sgnb.BATHY_SHOAL, bathy_par=shoal)
        x, y = node_coords(4, Nx, Ny, Lx, Ly, gll5())
        H = sgnb.setup_bathymetry(P=4, Nx=Nx, Ny=Ny, Lx=Lx, Ly=Ly, bathy_kind=sgnb.BATHY_SHOAL,
                                  bathy_par=shoal, bc_x=bc, bc_y=bc)["Hnod"]
        eta = 0.05 * np.exp(-((x - 0.3 * Lx) ** 2 + (y - 0.5 * Ly) ** 2) / (0.02 * Lx * Ly))
        z = np.zeros_like(x)
        out.append((kw, make_state(H + eta, 0.1 * np.sin(2 * np.pi * y / Ly) * (1 - bc),
                                   z, z, z)))
    return out


def single_runs(cases, dt0, nsteps):
    res = []
    for (kw, U), d0 in zip(cases, dt0):
        with sgnb.SGN2DB200(precision=sgnb.FP64_FAST, **kw) as d:
            d.upload(U)
            st = d.integrate_steps(0.0, d0, nsteps)
            res.append((d.download(), st))
    return res


def make_batch(cases):
    b = sgnb.SGNBatch([kw for kw, _ in cases])
    for i, (_, U) in enumerate(cases):
        b[i].upload(U)
    return b


def dt0_of(cases):
    out = []
    for kw, U in cases:
        with sgnb.SGN2DB200(precision=sgnb.FP64_FAST, **kw) as d:
            d.upload(U)
            out.append(d.cfl_time_step(0.5))
    return np.array(out)


def test_batch_matches_single_runs():
    cases = small_batch()
    dt0 = dt0_of(cases)
    ref = single_runs(cases, dt0, 15)
    with make_batch(cases) as b:
        assert b.config == (0, 0)
        stats = b.integrate_steps(dt0, 15)
        for i, (U1, st1) in enumerate(ref):
            assert rel_per_field(b[i].download(), U1) < 1e-10, f"instance {i}"
            st = stats[i]
            assert (st.accepted, st.rejected, st.rhsEvals) == \
                (st1.accepted, st1.rejected, st1.rhsEvals)
            assert abs(st.dtLast - st1.dtLast) <= 1e-10 * st1.dtLast
        # a second call continues from the states the first left
        stats2 = b.integrate_steps(dt0, 5)
        assert all(s.accepted == 5 for s in stats2)


@pytest.mark.parametrize("shape", [1, 2])
def test_batch_other_tile_shapes(shape):
    cases = small_batch(seed=11)
    dt0 = dt0_of(cases)
    ref = single_runs(cases, dt0, 12)
    with make_batch(cases) as b:
        b.config = (shape, 3 * 148)  # persistent grid; the default is one CTA per tile
        stats = b.integrate_steps(dt0, 12)
        for i, (U1, st1) in enumerate(ref):
            assert rel_per_field(b[i].download(), U1) < 1e-10, f"instance {i}"
            assert stats[i].accepted == 12 and stats[i].rejected == st1.rejected


def test_batch_against_oracle():
    cases = small_batch(seed=3)[:3]
    dt0 = dt0_of(cases)
    with make_batch(cases) as b:
        stats = b.integrate_steps(dt0, 8)
        for i, (kw, U) in enumerate(cases):
            o = O.Oracle(**kw)
            uo, so, _ = o.integrate_adaptive(U, 0.0, 1e300, dt0[i], stop_after=8)
            assert (stats[i].accepted, stats[i].rejected) == (so["accepted"], so["rejected"])
            assert rel_per_field(b[i].download(), uo) < 1e-10


def test_autotune_keeps_states():
    cases = small_batch(seed=5)
    dt0 = dt0_of(cases)
    with make_batch(cases) as b:
        before = [b[i].download() for i in range(len(b))]
        ms = b.autotune(dt0, reps=2)
        assert ms.shape == (3, 5) and np.all(ms > 0)
        shape, blocks = b.config
        assert ms[shape, blocks // 148] == ms.min()
        for i in range(len(b)):
            assert bits_equal(b[i].download(), before[i])
        b.integrate_steps(dt0, 3)


def test_nan_instance_isolated():
    cases = small_batch(seed=9)[:4]
    dt0 = dt0_of(cases)
    ref = single_runs(cases, dt0, 6)
    bad = cases[2][1].copy()
    bad[7] = np.nan
    with make_batch(cases) as b:
        b[2].upload(bad)
        with pytest.raises(sgnb.SgnbError) as ei:
            b.integrate_steps(dt0, 6)
        assert ei.value.status == 4
        for i in (0, 1, 3):
            assert rel_per_field(b[i].download(), ref[i][0]) < 1e-10


def test_sweep_generator_shapes():
    from sgnb import workloads as W

    inst = W.cfg4_instances()
    assert len(inst) == 256
    assert all(64 <= k["Nx"] <= 512 and 32 <= k["Ny"] <= 256 for k in inst)
    kw = dict(inst[0])
    kw.update(Nx=16, Ny=8)
    t = W.hump_shoal_state_torch(kw, device="cuda")
    with sgnb.SGN2DB200(precision=sgnb.FP64_FAST, **kw) as d:
        d.upload_tensor(t)
        x, y = d.node_coords()
        H = sgnb.setup_bathymetry(P=4, Nx=16, Ny=8, Lx=kw["Lx"], Ly=kw["Ly"], bathy_kind=3,
                                  bathy_par=kw["bathy_par"], bc_x=1, bc_y=1)["Hnod"]
        h = d.download()[: d.Nd]
        eta = 0.05 * np.exp(-((x - 6.0) ** 2 + (y - 5.0) ** 2) / 0.5)
        assert np.abs(h - (H + eta)).max() < 1e-14


def test_mixed_batch_matches_single_runs():
    """The mixed-precision batch (8x4 tiles) against mixed single-instance runs."""
    cases = small_batch(seed=13)
    dt0 = dt0_of(cases)
    ref = []
    for (kw, U), d0 in zip(cases, dt0):
        with sgnb.SGN2DB200(precision=sgnb.MIXED, **kw) as d:
            d.upload(U)
            st = d.integrate_steps(0.0, d0, 10)
            ref.append((d.download(), st))
    b = sgnb.SGNBatch([kw for kw, _ in cases], precision=sgnb.MIXED)
    with b:
        for i, (_, U) in enumerate(cases):
            b[i].upload(U)
        ms = b.autotune(dt0, reps=2)
        assert np.all(ms[0] > 0) and np.all(ms[1:] == -1.0) and b.config[0] == 0
        with pytest.raises(sgnb.SgnbError):
            b.config = (1, 0)
        for grid in (0, 2 * 148):
            for i, (_, U) in enumerate(cases):
                b[i].upload(U)
            b.config = (0, grid)
            stats = b.integrate_steps(dt0, 10)
            for i, (U1, st1) in enumerate(ref):
                assert rel_per_field(b[i].download(), U1) < 1e-6, f"instance {i}"
                assert stats[i].accepted == 10 and stats[i].rejected == st1.rejected
