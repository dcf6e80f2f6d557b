"""CPU oracle runs that tests farm out to worker processes (spawned, never forked, so that
no CUDA context is inherited): each is a plain function of picklable arguments."""
from __future__ import annotations

import numpy as np

import oracle as O
from cases import make_state


def gauge_trajectory(kw, means, eta0, dts, gauges):
    """eta at the gauge nodes after every frozen bs3Step (src/solver/rk.cpp:41-54) of the
    oracle, with the still depth given by element means (BATHY_CELLS) and h0 = H + eta0."""
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


def gauge_loss(args):
    """Squared gauge misfit of one oracle trajectory: args = (kw, means, eta0, dts, gauges,
    target)."""
    kw, means, eta0, dts, gauges, target = args
    return float(((gauge_trajectory(kw, means, eta0, dts, gauges) - target) ** 2).sum())
