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
  819,200 nodal values of eta0 against central differences on 8 seeded directions
  (relative 1e-6 at the best step of a sweep).
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
import sgnb
from sgnb import adjoint as ADJ
from sgnb import workloads as W
from cases import G, GAMMA, gll5, make_state, node_coords

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


def oracle_gauges(kw, means, eta0, dts, gauges):
    kw = dict(kw)
    kw["bathy_par"] = np.concatenate([[kw["Nx"], kw["Ny"], kw["Lx"], kw["Ly"]], means])
    o = O.Oracle(**kw)
    H = o.bathymetry()["Hnod"]
    z = np.zeros_like(H)
    U = make_state(H + eta0, z, z, z, z)
    out = []
    t = 0.0
    for dt in dts:
        U = o.bs3_step(U, t, dt)
        t += dt
        out.append(U[gauges] - H[gauges])
    return np.array(out)


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


def fd_sweep(loss_of, p0, d, adj, h0=0.4, n=19):
    """Relative errors of central differences along d over steps h0 / 2^k, k < n: the
    second-order stencil D2(h) = (L(p + h d) - L(p - h d)) / 2h and the fourth-order
    central stencil (4 D2(h) - D2(2h)) / 3."""
    errs = []
    prev = None
    for k in range(n):
        eps = h0 / 2 ** k
        d2 = (loss_of(*(a + eps * b for a, b in zip(p0, d))) -
              loss_of(*(a - eps * b for a, b in zip(p0, d)))) / (2 * eps)
        errs.append(abs(d2 - adj) / max(abs(d2), abs(adj)))
        if prev is not None:
            d4 = (4.0 * d2 - prev) / 3.0
            errs.append(abs(d4 - adj) / max(abs(d4), abs(adj)))
        prev = d2
    return errs


def test_config5_gradients():
    """Eight seeded directions: four in the element means (independent normal values per
    element) and four in eta0 (smooth random fields), on the frozen step sizes of the
    adaptive run; plus one direction of nodal white noise in eta0 on the same steps
    capped at 0.8 x the CFL-0.5 step. The adaptive controller takes some steps up to
    1.2 x the CFL-0.5 step, where grid-scale perturbations of the free surface grow: along
    the uncapped sequence finite differences of white noise in eta0 leave the linear
    range for steps above 1e-6, whatever the adjoint. The loss depends weakly on the
    bathymetry over 200 steps (directional derivatives of order 1e-11): second-order
    central differences are rounding-limited below steps of 1e-2 and truncation-limited
    above, so the sweep also forms the fourth-order central stencil."""
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
                    # large white-noise steps overflow by design (see the assert below)
                    with np.errstate(over="ignore", invalid="ignore"):
                        return float(((A.forward(m, e0) - target) ** 2).sum())

                zm, ze = np.zeros_like(gm), np.zeros_like(ge)
                if label == "adaptive":
                    dirs = [(rng.standard_normal(gm.size) * 0.01, ze) for _ in range(4)]
                    dirs += [(zm, 0.01 * smooth_random_field(x, y, cfg["Lx"], cfg["Ly"], rng))
                             for _ in range(4)]
                else:
                    dirs = [(zm, rng.standard_normal(ge.size) * 0.01)]
                for k, dv in enumerate(dirs):
                    adj = float(gm @ dv[0] + ge @ dv[1])
                    errs = fd_sweep(loss_of, p0, dv, adj)
                    # large steps of white noise overflow (NaN): the sweep keeps the rest
                    assert np.nanmin(errs) <= 1e-6, f"{label} direction {k}: errors {errs}"
