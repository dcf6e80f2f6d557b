"""x-slab decomposition on one device: the slabs' right-hand side and BS3(2) steps against
the whole mesh.

* right-hand side, exact mode: bit for bit the whole mesh's (and the oracle's) for 1, 2
  and 3 slabs, periodic and walls, including a bathymetry that is not symmetric across
  the periodic wrap;
* frozen step sizes (bs3Step replay): bit for bit the whole mesh's bs3_steps;
* adaptive steps: the same accepted / rejected sequence, states within 1e-10 relative per
  field (the error norm is summed over the slabs' partials in another order than over
  the whole mesh's tiles, which may change its last bits);
* the slab contexts refuse the whole-mesh integrators, the adjoint and mixed precision.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
import sgnb
from cases import ALPHA, GAMMA, G, bump_case, gll5, make_state, node_coords
from conftest import bits_equal, rel_per_field
from sgnb.slabs import SlabSolver

pytestmark = pytest.mark.gpu


def shoal_case(bc, Nx=11, Ny=6):
    """An off-centre shoal: the depth at x = 0 and x = Lx differs."""
    Lx, Ly = 0.5 * Nx, 0.6 * Ny
    shoal = (1.0, 0.6, 0.3 * Lx, 0.45 * Ly, 0.25 * Lx, 0.2 * Ly)
    kw = dict(P=4, Nx=Nx, Ny=Ny, Lx=Lx, Ly=Ly, g=G, gamma=GAMMA, c=ALPHA * np.sqrt(G),
              bc_x=bc, bc_y=bc, bathy_kind=sgnb.BATHY_SHOAL, bathy_par=shoal)
    x, y = node_coords(4, Nx, Ny, Lx, Ly, gll5())
    H = sgnb.setup_bathymetry(P=4, Nx=Nx, Ny=Ny, Lx=Lx, Ly=Ly, bathy_kind=sgnb.BATHY_SHOAL,
                              bathy_par=shoal, bc_x=bc, bc_y=bc)["Hnod"]
    eta = 0.04 * np.exp(-((x - 0.6 * Lx) ** 2 + (y - 0.5 * Ly) ** 2) / (0.03 * Lx * Ly))
    kx = 2 * np.pi / Lx
    U = make_state(H + eta, 0.05 * np.sin(kx * x) * (1 - bc), 0.02 * np.cos(kx * x) * (1 - bc),
                   0.01 * np.sin(kx * x), 0.005 * np.cos(kx * x))
    return kw, U


@pytest.mark.parametrize("bc", [0, 1])
@pytest.mark.parametrize("nslabs", [1, 2, 3])
@pytest.mark.parametrize("case", ["bump", "shoal"])
def test_rhs_bitwise(case, nslabs, bc):
    kw, U = bump_case(bc, Nx=10, Ny=6) if case == "bump" else shoal_case(bc)
    kw = dict(kw, precision=sgnb.FP64_EXACT)
    with sgnb.SGN2DB200(**kw) as d:
        R = d.rhs(U)
    assert bits_equal(R, O.Oracle(**{k: v for k, v in kw.items() if k != "precision"}).rhs(U))
    with SlabSolver(kw, nslabs=nslabs) as s:
        assert bits_equal(s.rhs(U), R)
        # upload / download round trip through the column scatter
        s.upload(U)
        assert bits_equal(s.download(), U)
        import torch

        s.upload_tensor(torch.from_numpy(U[::-1].copy()).cuda())
        assert bits_equal(s.download_tensor().cpu().numpy(), U[::-1])


@pytest.mark.parametrize("bc", [0, 1])
def test_frozen_replay_bitwise(bc):
    kw, U = shoal_case(bc, Nx=11, Ny=6)
    kw = dict(kw, precision=sgnb.FP64_EXACT)
    with sgnb.SGN2DB200(**kw) as d:
        d.upload(U)
        dt0 = d.cfl_time_step(0.4)
        n = 12
        dts = dt0 * (1.0 + 0.2 * np.sin(np.arange(n)))
        d.bs3_steps(0.0, dts)
        ref = d.download()
    with SlabSolver(kw, nslabs=3) as s:
        s.upload(U)
        st = s.integrate_steps(0.0, dts[0], n, dts=dts)
        assert st.accepted == n and st.rejected == 0
        assert bits_equal(s.download(), ref)


def test_adaptive_matches_whole_mesh():
    kw, U = bump_case(0, Nx=12, Ny=6)
    kw = dict(kw, precision=sgnb.FP64_FAST)
    with sgnb.SGN2DB200(**kw) as d:
        d.upload(U)
        dt0 = d.cfl_time_step(0.5)
        st1 = d.integrate_steps(0.0, dt0, 10)
        ref = d.download()
    for nslabs in (2, 3):
        with SlabSolver(kw, nslabs=nslabs) as s:
            s.upload(U)
            st = s.integrate_steps(0.0, dt0, 10, check_every=3)
            assert (st.accepted, st.rejected) == (st1.accepted, st1.rejected)
            assert abs(st.tReached - st1.tReached) <= 1e-12 * st1.tReached
            assert rel_per_field(s.download(), ref) < 1e-10


def test_nan_slab_stops_every_slab():
    kw, U = bump_case(1, Nx=12, Ny=6)
    kw = dict(kw, precision=sgnb.FP64_FAST)
    bad = U.copy()
    bad[5] = np.nan  # a node of the first slab
    with SlabSolver(kw, nslabs=3) as s:
        s.upload(bad)
        with pytest.raises(sgnb.SgnbError) as ei:
            s.integrate_steps(0.0, 1e-3, 5)
        assert ei.value.status == 4


def test_slab_contexts_refuse_whole_mesh_entries():
    kw, U = bump_case(0, Nx=10, Ny=6)
    kw = dict(kw, precision=sgnb.FP64_FAST)
    with SlabSolver(kw, nslabs=2) as s:
        ctx = s.slabs[0].ctx
        with pytest.raises(sgnb.SgnbError):
            ctx.integrate_steps(0.0, 1e-3, 2)
        with pytest.raises(sgnb.SgnbError):
            ctx.bs3_steps(0.0, [1e-3])
        with pytest.raises(sgnb.SgnbError):
            ctx.rk4_steps(0.0, [1e-3])
        from sgnb.adjoint import SGNAdjoint

        with pytest.raises(sgnb.SgnbError):
            SGNAdjoint(ctx, [1e-3], [0])
    with pytest.raises(sgnb.SgnbError):
        SlabSolver(dict(kw, precision=sgnb.MIXED), nslabs=2)


@pytest.mark.parametrize("bc", [0, 1])
def test_adaptive_to_end_time(bc):
    """integrateAdaptive to tEnd: the same attempts and end time as the whole mesh."""
    kw, U = shoal_case(bc, Nx=13, Ny=5)
    kw = dict(kw, precision=sgnb.FP64_FAST)
    with sgnb.SGN2DB200(**kw) as d:
        d.upload(U)
        dt0 = d.cfl_time_step(0.5)
        tEnd = 7.3 * dt0
        st1 = d.integrate_adaptive(0.0, tEnd, dt0)
        ref = d.download()
    with SlabSolver(kw, nslabs=3) as s:
        s.upload(U)
        st = s.integrate_adaptive(0.0, tEnd, dt0)
        assert (st.accepted, st.rejected, st.rhsEvals) == (st1.accepted, st1.rejected,
                                                           st1.rhsEvals)
        assert abs(st.tReached - tEnd) <= 1e-14 * tEnd and abs(st1.tReached - tEnd) <= 1e-14 * tEnd
        assert rel_per_field(s.download(), ref) < 1e-10
        # a run that starts at its end time takes no step
        st0 = s.integrate_adaptive(tEnd, tEnd, dt0)
        assert st0.accepted == 0 and st0.rejected == 0


# ---------------------------------------------------------------------------- fused exchange
from sgnb.slabs import PeerSlabSolver  # noqa: E402


@pytest.mark.parametrize("streams", ["shared", "per-slab"])
@pytest.mark.parametrize("bc", [0, 1])
@pytest.mark.parametrize("nslabs", [1, 2, 3, 4])
def test_fused_exchange_frozen_replay_bitwise(streams, bc, nslabs):
    """Stage kernels storing the next stage's edge inputs into the neighbours' ghosts, the
    controller reading all slabs' partials in place: the whole mesh's bs3 steps bit for
    bit, with every slab on one stream or each on its own (concurrent) stream."""
    kw, U = shoal_case(bc, Nx=13, Ny=6)
    kw = dict(kw, precision=sgnb.FP64_EXACT)
    with sgnb.SGN2DB200(**kw) as d:
        d.upload(U)
        R = d.rhs(U)
        dt0 = d.cfl_time_step(0.4)
        n = 9
        dts = dt0 * (1.0 + 0.2 * np.cos(np.arange(n)))
        d.bs3_steps(0.0, dts)
        ref = d.download()
    with PeerSlabSolver(kw, nslabs=nslabs, streams=streams) as s:
        assert bits_equal(s.rhs(U), R)
        s.upload(U)
        st = s.integrate_steps(0.0, dts[0], n, dts=dts, check_every=2)
        assert st.accepted == n and st.rejected == 0
        assert bits_equal(s.download(), ref)


@pytest.mark.parametrize("streams", ["shared", "per-slab"])
def test_fused_exchange_adaptive(streams):
    kw, U = bump_case(1, Nx=16, Ny=6)
    kw = dict(kw, precision=sgnb.FP64_FAST)
    with sgnb.SGN2DB200(**kw) as d:
        d.upload(U)
        dt0 = d.cfl_time_step(0.5)
        tEnd = 11.5 * dt0
        st1 = d.integrate_adaptive(0.0, tEnd, dt0)
        ref = d.download()
    with PeerSlabSolver(kw, nslabs=4, streams=streams) as s:
        s.upload(U)
        st = s.integrate_adaptive(0.0, tEnd, dt0, check_every=3)
        assert (st.accepted, st.rejected) == (st1.accepted, st1.rejected)
        assert abs(st.tReached - tEnd) <= 1e-14 * tEnd
        assert rel_per_field(s.download(), ref) < 1e-10
