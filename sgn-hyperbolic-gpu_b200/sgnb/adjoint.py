"""Adjoint of a frozen-dt BS3(2) trajectory: gauge records of the free surface and their
vector-Jacobian product (the sgnb_adj_* entry points), plus the torch.autograd.Function
that exposes them to a torch loss.

The trajectory is parameterised by the bathymetry as Nx * Ny element means (mapped to the
depth statics by the bilinear cell interpolant, BATHY_CELLS with Mx = Nx, My = Ny) and the
initial free surface eta0 (one value per node; h0 = H + eta0, zero velocity, w = p = 0).
The solver context passed in supplies the mesh, the physical parameters, the boundaries
and the arithmetic mode (FP64_FAST or FP64_EXACT); the forward run replaces its
bathymetry and leaves the final state in it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import SGN2DB200, _check, _ptr, lib


class SGNAdjoint:
    def __init__(self, solver: SGN2DB200, dts, gauge_nodes, checkpoint_every: int = 20):
        self.solver = solver
        self.dts = np.ascontiguousarray(dts, dtype=np.float64)
        self.gauges = np.ascontiguousarray(gauge_nodes, dtype=np.int64)
        self.N, self.ng = int(self.dts.size), int(self.gauges.size)
        self.generation = 0
        h = C.c_void_p()
        _check(lib().sgnb_adj_create(solver._h, self.N, _ptr(self.dts), self.ng,
                                     self.gauges.ctypes.data_as(C.POINTER(C.c_longlong)),
                                     int(checkpoint_every), C.byref(h)), solver._h)
        self._a = h

    def close(self):
        if getattr(self, "_a", None):
            lib().sgnb_adj_destroy(self._a)
            self._a = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def forward(self, means, eta0) -> np.ndarray:
        """Runs the trajectory; returns eta at the gauges after every step, [N, ngauges]."""
        m = np.ascontiguousarray(means, dtype=np.float64).reshape(-1)
        e = np.ascontiguousarray(eta0, dtype=np.float64).reshape(-1)
        if m.size != self.solver.Nx * self.solver.Ny or e.size != self.solver.Nd:
            raise ValueError("means: Nx * Ny values, eta0: nDof values")
        out = np.zeros((self.N, max(self.ng, 1)))
        _check(lib().sgnb_adj_forward(self._a, _ptr(m), _ptr(e), _ptr(out)), self.solver._h)
        self.generation += 1
        return out[:, : self.ng]

    def vjp(self, eta_bar):
        """Gradients (element means, eta0) of <eta_bar, eta> for the last forward run."""
        eb = np.ascontiguousarray(eta_bar, dtype=np.float64).reshape(-1)
        if eb.size != self.N * self.ng:
            raise ValueError("eta_bar: [nsteps, ngauges] values")
        gm = np.zeros(self.solver.Nx * self.solver.Ny)
        ge = np.zeros(self.solver.Nd)
        if eb.size == 0:
            eb = np.zeros(1)
        _check(lib().sgnb_adj_vjp(self._a, _ptr(eb), _ptr(gm), _ptr(ge)), self.solver._h)
        return gm, ge


def gauge_trajectory():
    """The torch.autograd.Function (built lazily so that importing sgnb needs no torch)."""
    import torch

    class GaugeTrajectory(torch.autograd.Function):
        """eta[N, ngauges] = trajectory(means, eta0); backward through sgnb_adj_vjp."""

        @staticmethod
        def forward(ctx, means, eta0, adj: SGNAdjoint):
            eta = adj.forward(means.detach().cpu().double().numpy(),
                              eta0.detach().cpu().double().numpy())
            ctx.adj = adj
            ctx.generation = adj.generation
            ctx.dev = means.device
            return torch.from_numpy(eta).to(means.device)

        @staticmethod
        def backward(ctx, eta_bar):
            if ctx.adj.generation != ctx.generation:
                raise RuntimeError("GaugeTrajectory: another forward ran on this SGNAdjoint "
                                   "since this graph was built")
            gm, ge = ctx.adj.vjp(eta_bar.detach().cpu().double().numpy())
            return (torch.from_numpy(gm).to(ctx.dev), torch.from_numpy(ge).to(ctx.dev), None)

    return GaugeTrajectory
