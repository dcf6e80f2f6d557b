"""Workload definitions: the benchmark configurations as solver arguments plus a state.

Configuration 2 (the benchmark workload): 2048 x 1024 elements, P = 4, on a 40 x 20 basin
with reflective walls. Still depth: a 0.45 plane with an elliptic shoal centred at
(20, 10), semi-axes 4 (x) and 3 (y), crest depth 0.15, profile
H = 0.45 - 0.30 (1 - r^2)^3 inside the ellipse. Free surface: the sum of 8 sine waves with
seeded random phase, direction, amplitude in [0.005, 0.02] and wavelength in [1, 4]
(numpy default_rng(2)); zero initial velocity, w = p = 0. alpha = 3 with c = alpha sqrt(g H0),
H0 = 0.45; gamma = 1.5. 500 adaptive BS3(2) steps, atol 1e-8, rtol 1e-6.

States are built in float64 with torch on the device (fast at 52M nodes) or with numpy on
the host; the two agree to libm rounding, and each run feeds one state to every solver it
compares.
"""
from __future__ import annotations

import math

import numpy as np

G, GAMMA, ALPHA = 9.81, 1.5, 3.0
CFG2 = dict(Nx=2048, Ny=1024, Lx=40.0, Ly=20.0, steps=500)


def cfg2_params(seed: int = 2):
    """Depth profile (BATHY_SHOAL parameters) and the 8 wave components."""
    shoal = (0.45, 0.15, 20.0, 10.0, 4.0, 3.0)
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.005, 0.02, 8)
    lam = rng.uniform(1.0, 4.0, 8)
    theta = rng.uniform(0.0, 2 * np.pi, 8)
    phase = rng.uniform(0.0, 2 * np.pi, 8)
    return shoal, (amp, lam, theta, phase)


def cfg2_solver_args(Nx=2048, Ny=1024, Lx=40.0, Ly=20.0, seed=2):
    shoal, _ = cfg2_params(seed)
    return dict(P=4, Nx=Nx, Ny=Ny, Lx=Lx, Ly=Ly, g=G, c=ALPHA * math.sqrt(G * shoal[0]),
                gamma=GAMMA, bc_x=1, bc_y=1, bathy_kind=3, bathy_par=shoal)


def cfg2_state_torch(Nx=2048, Ny=1024, Lx=40.0, Ly=20.0, seed=2, device="cuda"):
    """Initial state of configuration 2 as a float64 torch tensor (var-major layout)."""
    import torch

    shoal, (amp, lam, theta, phase) = cfg2_params(seed)
    s = math.sqrt(3.0 / 7.0)
    nodes = torch.tensor([-1.0, -s, 0.0, s, 1.0], dtype=torch.float64, device=device)
    hx, hy = Lx / Nx, Ly / Ny
    a = torch.arange(5, device=device).repeat(5)
    b = torch.arange(5, device=device).repeat_interleave(5)
    U = torch.zeros(5, Ny, Nx, 25, dtype=torch.float64, device=device)
    ex = torch.arange(Nx, device=device, dtype=torch.float64)
    for r0 in range(0, Ny, 64):  # bounded temporaries
        ey = torch.arange(r0, min(r0 + 64, Ny), device=device, dtype=torch.float64)
        x = (ex[None, :, None] * hx + 0.5 * hx * (nodes[a][None, None, :] + 1.0))
        y = (ey[:, None, None] * hy + 0.5 * hy * (nodes[b][None, None, :] + 1.0))
        x, y = torch.broadcast_tensors(x, y)
        dx, dy = (x - shoal[2]) / shoal[4], (y - shoal[3]) / shoal[5]
        q = torch.clamp(1.0 - (dx * dx + dy * dy), min=0.0)
        H = shoal[0] - (shoal[0] - shoal[1]) * q ** 3
        eta = torch.zeros_like(x)
        for A, L, T, P in zip(amp, lam, theta, phase):
            k = 2 * math.pi / L
            eta += A * torch.sin(k * (x * math.cos(T) + y * math.sin(T)) + P)
        U[0, r0:r0 + ey.numel()] = H + eta
    return U.reshape(-1)


# ---------------------------------------------------------------------------------------
# Configuration 4: the batched sweep. 256 instances (numpy default_rng(4)), each on the
# 20 x 10 basin with reflective walls: Nx ~ U{64..512} and Ny ~ U{32..256} drawn
# independently, alpha ~ U[1.5, 6] (c = alpha sqrt(g H0)), still depth a 1.0 plane with an
# elliptic shoal centred at (12, 5), semi-axes 4 x 3, crest depth ~ U[0.3, 0.9]
# (BATHY_SHOAL profile). Incident wave: the Gaussian hump of configuration 1,
# eta = 0.05 exp(-((x - 6)^2 + (y - 5)^2) / 0.5), placed up-slope of the shoal; zero velocity,
# w = p = 0.
# ---------------------------------------------------------------------------------------
CFG4 = dict(n=256, Lx=20.0, Ly=10.0, H0=1.0, seed=4)


def cfg4_instances(n=256, seed=4, nx_range=(64, 512), ny_range=(32, 256)):
    """Solver keyword dicts of the sweep's instances (FP64_FAST, walls)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        Nx = int(rng.integers(nx_range[0], nx_range[1] + 1))
        Ny = int(rng.integers(ny_range[0], ny_range[1] + 1))
        alpha = float(rng.uniform(1.5, 6.0))
        crest = float(rng.uniform(0.3, 0.9))
        shoal = (CFG4["H0"], crest, 12.0, 5.0, 4.0, 3.0)
        out.append(dict(P=4, Nx=Nx, Ny=Ny, Lx=CFG4["Lx"], Ly=CFG4["Ly"], g=G,
                        c=alpha * math.sqrt(G * CFG4["H0"]), gamma=GAMMA, bc_x=1, bc_y=1,
                        bathy_kind=3, bathy_par=shoal))
    return out


def hump_shoal_state_torch(kw, device="cuda"):
    """Initial state of one sweep instance as a float64 torch tensor (var-major)."""
    import torch

    Nx, Ny, Lx, Ly = kw["Nx"], kw["Ny"], kw["Lx"], kw["Ly"]
    shoal = kw["bathy_par"]
    s = math.sqrt(3.0 / 7.0)
    nodes = torch.tensor([-1.0, -s, 0.0, s, 1.0], dtype=torch.float64, device=device)
    hx, hy = Lx / Nx, Ly / Ny
    a = torch.arange(5, device=device).repeat(5)
    b = torch.arange(5, device=device).repeat_interleave(5)
    ex = torch.arange(Nx, device=device, dtype=torch.float64)
    ey = torch.arange(Ny, device=device, dtype=torch.float64)
    x = ex[None, :, None] * hx + 0.5 * hx * (nodes[a][None, None, :] + 1.0)
    y = ey[:, None, None] * hy + 0.5 * hy * (nodes[b][None, None, :] + 1.0)
    x, y = torch.broadcast_tensors(x, y)
    dx, dy = (x - shoal[2]) / shoal[4], (y - shoal[3]) / shoal[5]
    q = torch.clamp(1.0 - (dx * dx + dy * dy), min=0.0)
    H = shoal[0] - (shoal[0] - shoal[1]) * q ** 3
    eta = 0.05 * torch.exp(-((x - 6.0) ** 2 + (y - 5.0) ** 2) / 0.5)
    U = torch.zeros(5, Ny, Nx, 25, dtype=torch.float64, device=device)
    U[0] = H + eta
    return U.reshape(-1)


# ---------------------------------------------------------------------------------------
# Configuration 5: the adjoint. 256 x 128 elements on the 20 x 10 basin with reflective
# walls, alpha = 3 (c = 3 sqrt(g)), FP64. Bathymetry: 32,768 element means, the elliptic
# shoal of configuration 4 (plane 1.0, crest 0.5 at (12, 5), semi-axes 4 x 3) sampled at
# the element centres plus seeded noise of standard deviation 0.005 (numpy
# default_rng(5)); mapped to the nodes by the bilinear cell interpolant (BATHY_CELLS).
# Initial free surface: the Gaussian hump 0.05 exp(-((x - 6)^2 + (y - 5)^2) / 0.5).
# 16 gauges at the nearest nodes of seeded uniform positions. Target: the run from means
# perturbed by seeded noise of standard deviation 0.01 and a hump 10 % higher. The 200
# step sizes come from an adaptive run of the unperturbed problem (atol 1e-8, rtol 1e-6)
# and are then frozen; checkpoints every 20 steps.
# ---------------------------------------------------------------------------------------
CFG5 = dict(Nx=256, Ny=128, Lx=20.0, Ly=10.0, steps=200, gauges=16, checkpoint=20, seed=5)


def gll_nodes():
    s = math.sqrt(3.0 / 7.0)
    return np.array([-1.0, -s, 0.0, s, 1.0])


def node_coords_np(Nx, Ny, Lx, Ly):
    """Node coordinates in the solver's layout (e * 25 + a + 5 b), numpy."""
    xi = gll_nodes()
    hx, hy = Lx / Nx, Ly / Ny
    a = np.tile(np.arange(5), 5)
    b = np.repeat(np.arange(5), 5)
    ex = np.arange(Nx)
    ey = np.arange(Ny)
    x = ex[None, :, None] * hx + 0.5 * hx * (xi[a][None, None, :] + 1.0)
    y = ey[:, None, None] * hy + 0.5 * hy * (xi[b][None, None, :] + 1.0)
    x, y = np.broadcast_arrays(x, y)
    return x.reshape(-1).copy(), y.reshape(-1).copy()


def cfg5_problem(Nx=256, Ny=128, Lx=20.0, Ly=10.0, ngauges=16, seed=5):
    """Means, eta0, gauge nodes, the target's parameters and the solver arguments."""
    rng = np.random.default_rng(seed)
    cx = (np.arange(Nx) + 0.5) * Lx / Nx
    cy = (np.arange(Ny) + 0.5) * Ly / Ny
    X, Y = np.meshgrid(cx, cy)
    r2 = ((X - 12.0) / 4.0) ** 2 + ((Y - 5.0) / 3.0) ** 2
    q = np.clip(1.0 - r2, 0.0, None)
    means = (1.0 - 0.5 * q ** 3 + 0.005 * rng.standard_normal(X.shape)).reshape(-1)
    x, y = node_coords_np(Nx, Ny, Lx, Ly)
    eta0 = 0.05 * np.exp(-((x - 6.0) ** 2 + (y - 5.0) ** 2) / 0.5)
    gx = rng.uniform(0.0, Lx, ngauges)
    gy = rng.uniform(0.0, Ly, ngauges)
    gauges = np.array([int(np.argmin((x - px) ** 2 + (y - py) ** 2)) for px, py in zip(gx, gy)],
                      dtype=np.int64)
    target_means = means + 0.01 * rng.standard_normal(means.shape)
    target_eta0 = 1.1 * eta0
    kw = dict(P=4, Nx=Nx, Ny=Ny, Lx=Lx, Ly=Ly, g=G, c=ALPHA * math.sqrt(G * 1.0), gamma=GAMMA,
              bc_x=1, bc_y=1, bathy_kind=5, bathy_par=np.concatenate([[Nx, Ny, Lx, Ly], means]))
    return dict(kw=kw, means=means, eta0=eta0, gauges=gauges, target_means=target_means,
                target_eta0=target_eta0)
