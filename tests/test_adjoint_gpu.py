"""The adjoint: hand-written VJP kernels of the right-hand side and of the BS3(2) update.

* right-hand side: <Rbar, dR[dU, dS]> from central differences of the CPU oracle's rhs
  equals <Ubar, dU> + sum <Sbar_k, dS_k> from sgnb_rhs_vjp, for the state and for each
  depth static separately (nodal H, dH/dx, dH/dy, face depths, wall-edge depths), with
  periodic boundaries and with walls (relative 1e-6);
* trajectory: the device forward (frozen step sizes, gauges, checkpoints) follows the
  oracle's bs3 steps (1e-10), the torch.autograd.Function gives sgnb_adj_vjp's
  gradients, and directional derivatives of the gauge-misfit loss agree with central
  differences of the device forward and of the oracle's forward (relative 1e-6);
* configuration 5 (256 x 128, 200 frozen steps from an adaptive run, 16 gauges,
  checkpoints every 20 steps): gradients with respect to the 32,768 element means and the
  819,200 nodal values of eta0 against central differences of the device forward on 8
  seeded directions plus a white-noise one, and of the CPU oracle's forward on two of them,
  each with a stencil and step fixed in advance (relative 1e-6).
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
import sgnb
from sgnb import adjoint as ADJ
from sgnb import workloads as W
from cases import G, GAMMA, gll5, make_state, node_coords
import oracle_runs

pytestmark = pytest.mark.gpu

STATICS = ("Hnod", "Hx", "Hy", "HfaceX", "HfaceY", "HfaceXEnd", "HfaceYEnd")


def rhs_case(bc, Nx=6, Ny=5, seed=0):
    Lx, Ly = 6.0, 5.0
    bump = (1.0, 0.3, 3.1, 2.4, 3.0)
    kw = dict(P=4, Nx=Nx, Ny=Ny, Lx=Lx, Ly=Ly, g=G, c=3.0 * np.sqrt(G), gamma=GAMMA, bc_x=bc,
              bc_y=bc, bathy_kind=sgnb.BATHY_GAUSS, bathy_par=bump)
    x, y = node_coords(4, Nx, Ny, Lx, Ly, gll5())
    H = sgnb.setup_bathymetry(P=4, Nx=Nx, Ny=Ny, Lx=Lx, Ly=Ly, bathy_kind=sgnb.BATHY_GAUSS,
                              bathy_par=bump, bc_x=bc, bc_y=bc)["Hnod"]
    kx, ky = 2 * np.pi / Lx, 2 * np.pi / Ly
    h = H + 0.05 * np.sin(kx * x + 0.3) * np.cos(ky * y)
    U = make_state(h, 0.3 + 0.1 * np.sin(ky * y), -0.2 + 0.1 * np.cos(kx * x),
                   0.05 * np.cos(kx * x + ky * y), 0.02 * np.sin(kx * x - ky * y))
    return kw, U


def oracle_rhs(o, U, S):
    o.set_bathymetry(S)
    return o.rhs(U)


@pytest.mark.parametrize("bc,manning", [(sgnb.BC_PERIODIC, 0.0), (sgnb.BC_WALL, 0.0),
                                        (sgnb.BC_WALL, 0.03)])
def test_rhs_vjp_against_oracle_differences(bc, manning):
    kw, U = rhs_case(bc)
    kw = dict(kw, nManning=manning)
    rng = np.random.default_rng(10 + bc)
    o = O.Oracle(**kw)
    S0 = o.bathymetry()
    Rbar = rng.standard_normal(U.size)
    with sgnb.SGN2DB200(precision=sgnb.FP64_FAST, **kw) as d:
        Ub, Sb = d.rhs_vjp(U, Rbar)
    eps = 1e-6
    checks = [("U", rng.standard_normal(U.size) * np.repeat([0.05, 0.05, 0.05, 0.02, 0.02],
                                                           U.size // 5))]
    for k in STATICS:
        checks.append((k, rng.standard_normal(S0[k].size) * 0.05))
    for name, dv in checks:
        if name == "U":
            Rp = oracle_rhs(o, U + eps * dv, S0)
            Rm = oracle_rhs(o, U - eps * dv, S0)
            adj = float(Ub @ dv)
        else:
            Sp = dict(S0); Sp[name] = S0[name] + eps * dv
            Sm = dict(S0); Sm[name] = S0[name] - eps * dv
            Rp = oracle_rhs(o, U, Sp)
            Rm = oracle_rhs(o, U, Sm)
            adj = float(Sb[name] @ dv)
        fd = float(Rbar @ ((Rp - Rm) / (2 * eps)))
        scale = max(abs(fd), abs(adj), 1e-3 * np.abs(Rbar).sum() * 0.05)
        if name in ("HfaceXEnd", "HfaceYEnd") and bc == sgnb.BC_PERIODIC:
            assert adj == 0.0 and abs(fd) < 1e-8, name  # unused without walls
            continue
        assert abs(fd - adj) <= 1e-6 * scale, f"{name}: fd {fd:.12e} adjoint {adj:.12e}"
    o.set_bathymetry(S0)


def small_problem(Nx=12, Ny=6, Lx=12.0, Ly=6.0, seed=4, ng=5):
    rng = np.random.default_rng(seed)
    cx = (np.arange(Nx) + 0.5) * Lx / Nx
    cy = (np.arange(Ny) + 0.5) * Ly / Ny
    X, Y = np.meshgrid(cx, cy)
    means = (1.0 - 0.3 * np.exp(-((X - 7.0) ** 2 + (Y - 3.0) ** 2) / 4.0)
             + 0.01 * rng.standard_normal(X.shape)).reshape(-1)
    kw = dict(P=4, Nx=Nx, Ny=Ny, Lx=Lx, Ly=Ly, g=G, c=3.0 * np.sqrt(G), gamma=GAMMA, bc_x=1,
              bc_y=1, bathy_kind=sgnb.BATHY_CELLS,
              bathy_par=np.concatenate([[Nx, Ny, Lx, Ly], means]))
    x, y = node_coords(4, Nx, Ny, Lx, Ly, gll5())
    eta0 = 0.05 * np.exp(-((x - 4.0) ** 2 + (y - 3.0) ** 2) / 1.0)
    gauges = rng.choice(x.size, ng, replace=False).astype(np.int64)
    return kw, means, eta0, gauges, rng


oracle_gauges = oracle_runs.gauge_trajectory


def test_trajectory_gradient_small():
    import torch

    kw, means, eta0, gauges, rng = small_problem()
    with sgnb.SGN2DB200(precision=sgnb.FP64_FAST, **kw) as d:
        H = sgnb.setup_bathymetry(**{k: kw[k] for k in ("P", "Nx", "Ny", "Lx", "Ly", "bc_x",
                                                       "bc_y", "bathy_kind", "bathy_par")})["Hnod"]
        z = np.zeros_like(H)
        d.upload(make_state(H + eta0, z, z, z, z))
        dt0 = d.cfl_time_step(0.4)
        dts = dt0 * (1.0 + 0.1 * np.sin(np.arange(24)))
        with ADJ.SGNAdjoint(d, dts, gauges, checkpoint_every=7) as A:
            eta = A.forward(means, eta0)
            ref = oracle_gauges(kw, means, eta0, dts, gauges)
            assert np.abs(eta - ref).max() <= 1e-10 * np.abs(ref).max()
            target = eta + 0.01 * rng.standard_normal(eta.shape)

            def loss_of(m, e0):
                return float(((A.forward(m, e0) - target) ** 2).sum())

            # autograd.Function against the direct vjp
            GT = ADJ.gauge_trajectory()
            mt = torch.tensor(means, requires_grad=True)
            et = torch.tensor(eta0, requires_grad=True)
            L = ((GT.apply(mt, et, A) - torch.from_numpy(target)) ** 2).sum()
            L.backward()
            gm, ge = A.vjp(2.0 * (A.forward(means, eta0) - target))
            assert np.array_equal(mt.grad.numpy(), gm) and np.array_equal(et.grad.numpy(), ge)
            # directional derivatives against central differences of the device forward
            for k in range(4):
                dm = rng.standard_normal(means.size) * 0.01
                de = rng.standard_normal(eta0.size) * 0.01
                adj = float(gm @ dm + ge @ de)
                errs = []
                for eps in (1e-3, 1e-4, 1e-5):
                    fd = (loss_of(means + eps * dm, eta0 + eps * de) -
                          loss_of(means - eps * dm, eta0 - eps * de)) / (2 * eps)
                    errs.append(abs(fd - adj) / max(abs(fd), abs(adj)))
                assert min(errs) <= 1e-6, f"direction {k}: relative errors {errs}"
            # and central differences of the oracle's (CPU) forward along one direction
            dm = rng.standard_normal(means.size) * 0.01
            de = rng.standard_normal(eta0.size) * 0.01
            eps = 1e-4
            Lp = float(((oracle_gauges(kw, means + eps * dm, eta0 + eps * de, dts, gauges)
                         - target) ** 2).sum())
            Lm = float(((oracle_gauges(kw, means - eps * dm, eta0 - eps * de, dts, gauges)
                         - target) ** 2).sum())
            fd = (Lp - Lm) / (2 * eps)
            adj = float(gm @ dm + ge @ de)
            assert abs(fd - adj) <= 1e-6 * max(abs(fd), abs(adj))


def smooth_random_field(x, y, Lx, Ly, rng, n=12, kmax=4):
    """Sum of n seeded Fourier modes with wavenumbers up to kmax per direction."""
    f = np.zeros_like(x)
    for _ in range(n):
        kx, ky = rng.integers(0, kmax + 1, 2) * 2 * np.pi / np.array([Lx, Ly])
        f += rng.standard_normal() * np.cos(kx * x + ky * y + rng.uniform(0, 2 * np.pi))
    return f / np.sqrt(n)


# Central-difference stencils and steps for configuration 5, fixed from a sweep over
# h = 0.4 / 2^k, k < 19, of the same seeded directions (second-order stencil D2(h) and the
# fourth-order (4 D2(h) - D2(2h)) / 3 at each step):
# * element-mean directions: the loss depends weakly on the bathymetry over 200 steps
#   (directional derivatives 3e-12 to 6e-11), so D2 is truncation-limited above h ~ 1e-2
#   and rounding-limited below, where the weakest direction's error jumps between 1e-7 and
#   1e-5 from one step to the next (and moves when the step sequence changes in its last
#   bits); the fourth-order stencil at h = 0.1, in the middle of the plateau, is within
#   1.9e-7 of the adjoint on all four (within 3.5e-7 at h = 0.05 and 0.2);
# * eta0 directions (smooth fields, and the white-noise field on the capped sequence): D2
#   at h = 0.4 / 2^15 = 1.22e-5 is within 4.1e-8 (2.2e-8 for the smooth ones).
H_MEANS = 0.1
H_ETA = 0.4 / 2 ** 15
FD_TOL = 1e-6


def d2(loss_of, p0, d, h):
    """Second-order central difference of loss_of along d at p0."""
    return (loss_of(*(a + h * b for a, b in zip(p0, d))) -
            loss_of(*(a - h * b for a, b in zip(p0, d)))) / (2 * h)


def d4(loss_of, p0, d, h):
    """Fourth-order central difference (4 D2(h) - D2(2h)) / 3."""
    return (4.0 * d2(loss_of, p0, d, h) - d2(loss_of, p0, d, 2 * h)) / 3.0


def rel(a, b):
    return abs(a - b) / max(abs(a), abs(b))


def test_config5_gradients():
    """Eight seeded directions, on the frozen step sizes of the adaptive run: four in the
    element means (independent normal values per element; fourth-order stencil at
    H_MEANS) and four in eta0 (smooth random fields; second-order stencil at H_ETA); plus
    one direction of nodal white noise in eta0 on the same steps capped at 0.8 x the
    CFL-0.5 step (second order at H_ETA). The adaptive controller takes some steps up to
    1.2 x the CFL-0.5 step, where grid-scale perturbations of the free surface grow: along
    the uncapped sequence finite differences of white noise in eta0 leave the linear range
    for steps above 1e-6, whatever the adjoint. Then the CPU oracle's forward (the
    reference algorithm restated, src/solver/rk.cpp:41-54 steps over src/solver/sgn2d.cpp
    right-hand sides) on the first element-mean and the first eta0 direction, with the
    same stencils: its central differences against the device adjoint, relative 1e-6.
    The oracle runs (about 45 s each on one core) go to spawned worker processes (never
    forked: a fork would copy this process's CUDA state)."""
    import multiprocessing as mp

    pool = mp.get_context("spawn").Pool(7)
    try:
        _config5_gradients(pool)
    finally:
        pool.close()
        pool.join()


def _config5_gradients(pool):
    P = W.cfg5_problem()
    kw = P["kw"]
    cfg = W.CFG5
    rng = np.random.default_rng(55)
    with sgnb.SGN2DB200(precision=sgnb.FP64_FAST, **kw) as d:
        H = sgnb.setup_bathymetry(**{k: kw[k] for k in ("P", "Nx", "Ny", "Lx", "Ly", "bc_x",
                                                       "bc_y", "bathy_kind", "bathy_par")})["Hnod"]
        z = np.zeros_like(H)
        d.upload(make_state(H + P["eta0"], z, z, z, z))
        dt0 = d.cfl_time_step(0.5)
        st = d.integrate_steps(0.0, dt0, cfg["steps"])
        log = d.attempt_log()
        dts = log[log[:, 3] == 1][:, 1].copy()
        assert dts.size == cfg["steps"] and st.accepted == cfg["steps"]
        x, y = W.node_coords_np(cfg["Nx"], cfg["Ny"], cfg["Lx"], cfg["Ly"])
        p0 = (P["means"], P["eta0"])
        for label, dl in (("adaptive", dts), ("capped", np.minimum(dts, 0.8 * dt0))):
            with ADJ.SGNAdjoint(d, dl, P["gauges"], checkpoint_every=cfg["checkpoint"]) as A:
                target = A.forward(P["target_means"], P["target_eta0"])
                eta = A.forward(*p0)
                assert eta.shape == (cfg["steps"], cfg["gauges"])
                gm, ge = A.vjp(2.0 * (eta - target))
                assert gm.shape == (cfg["Nx"] * cfg["Ny"],) and ge.shape == (d.Nd,)

                def loss_of(m, e0):
                    return float(((A.forward(m, e0) - target) ** 2).sum())

                zm, ze = np.zeros_like(gm), np.zeros_like(ge)
                if label == "adaptive":
                    dirs = [(rng.standard_normal(gm.size) * 0.01, ze) for _ in range(4)]
                    dirs += [(zm, 0.01 * smooth_random_field(x, y, cfg["Lx"], cfg["Ly"], rng))
                             for _ in range(4)]
                else:
                    dirs = [(zm, rng.standard_normal(ge.size) * 0.01)]
                errs = []
                for k, dv in enumerate(dirs):
                    adj = float(gm @ dv[0] + ge @ dv[1])
                    means_dir = label == "adaptive" and k < 4
                    fd = d4(loss_of, p0, dv, H_MEANS) if means_dir else d2(loss_of, p0, dv, H_ETA)
                    errs.append(rel(fd, adj))
                print(f"{label}: relative errors of the device forward's central differences",
                      " ".join(f"{e:.1e}" for e in errs))
                assert max(errs) <= FD_TOL, (label, errs)
                if label != "adaptive":
                    continue
                # the CPU oracle's forward along direction 0 (means) and 4 (eta0)
                pts = [(0, s_ * H_MEANS) for s_ in (1, -1, 2, -2)] + [(4, s_ * H_ETA) for s_ in (1, -1)]
                jobs = [(kw, P["target_means"], P["target_eta0"], dl, P["gauges"])]
                jobs += [(kw, p0[0] + h * dirs[k][0], p0[1] + h * dirs[k][1], dl, P["gauges"])
                         for k, h in pts]
                trajs = pool.starmap(oracle_runs.gauge_trajectory, jobs)
                L = {pt: float(((tr - trajs[0]) ** 2).sum()) for pt, tr in zip(pts, trajs[1:])}
                c2 = lambda k, h: (L[(k, h)] - L[(k, -h)]) / (2 * h)
                fd0 = (4.0 * c2(0, H_MEANS) - c2(0, 2 * H_MEANS)) / 3.0
                fd4 = c2(4, H_ETA)
                e0 = rel(fd0, float(gm @ dirs[0][0]))
                e4 = rel(fd4, float(ge @ dirs[4][1]))
                print(f"oracle central differences against the adjoint: means {e0:.1e}, "
                      f"eta0 {e4:.1e}")
                assert e0 <= FD_TOL and e4 <= FD_TOL
