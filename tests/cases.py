"""Test and benchmark cases: solver arguments plus initial states (numpy, var-major).

Each case returns ``(kwargs, U)`` where kwargs are the solver arguments shared by the
oracle (oracle/oracle.py) and the device solver (sgnb.SGN2DB200), and U is the initial
state in the reference layout. The same U array is fed to every implementation, so the
state's own round-off is irrelevant to parity.

Cases:
  bump_case     the GPU parity case of the reference (test/test_cuda_sgn2d.cu:38-64)
  lake_case     lake at rest over the same bump (test/test_sgn2d.cpp:55-66)
  gauss_case    Gauss-Legendre solution points (PointSet::GaussLegendre): flat bottom
                H = 0, which SGN2D requires for them (sgn2d.cpp:46-47), smooth state
  cfg1_case     configuration 1: 128x64 on 20x10, flat depth 1, Gaussian hump of 0.05
  cfg2_case     configuration 2: 2048x1024 on 40x20 with reflective walls, 0.45 plane with
                an elliptic shoal (semi-axes 4 x 3, crest depth 0.15, centred), and 8
                seeded random-phase sine waves (amplitude 0.005-0.02, wavelength 1-4),
                zero initial velocity
"""
from __future__ import annotations

import numpy as np

G = 9.81
GAMMA = 1.5
ALPHA = 3.0
CFG1_STEPS = 100
CFG2_STEPS = 500

BC_PERIODIC, BC_WALL = 0, 1
BATHY_NONE, BATHY_CONST, BATHY_GAUSS, BATHY_SHOAL, BATHY_GAUSS_SUM, BATHY_CELLS = range(6)


def node_coords(P, Nx, Ny, Lx, Ly, nodes):
    """SGN2D::nodeCoords (src/solver/sgn2d.cpp:89-102), vectorised."""
    np_ = P + 1
    hx, hy = Lx / Nx, Ly / Ny
    e = np.arange(Nx * Ny)
    ex, ey = e % Nx, e // Nx
    a = np.tile(np.arange(np_), np_)
    b = np.repeat(np.arange(np_), np_)
    x = (ex[:, None] * hx + 0.5 * hx * (nodes[a][None, :] + 1.0)).reshape(-1)
    y = (ey[:, None] * hy + 0.5 * hy * (nodes[b][None, :] + 1.0)).reshape(-1)
    return x, y


def gll5():
    """GLL nodes for P = 4 (closed form: 0, +-sqrt(3/7), +-1)."""
    s = np.sqrt(3.0 / 7.0)
    return np.array([-1.0, -s, 0.0, s, 1.0])


def gauss5():
    """Gauss-Legendre nodes for P = 4 (the roots of L_5, closed form)."""
    r = np.sqrt(5.0 - 2.0 * np.sqrt(10.0 / 7.0)) / 3.0
    s = np.sqrt(5.0 + 2.0 * np.sqrt(10.0 / 7.0)) / 3.0
    return np.array([-s, -r, 0.0, r, s])


def gauss_case(bc=BC_PERIODIC, Nx=8, Ny=6, Lx=10.0, Ly=8.0):
    c = ALPHA * np.sqrt(G * 1.0)
    kw = dict(P=4, Nx=Nx, Ny=Ny, Lx=Lx, Ly=Ly, g=G, c=c, gamma=GAMMA, bc_x=bc, bc_y=bc,
              bathy_kind=BATHY_NONE, bathy_par=(), points=1)
    x, y = node_coords(4, Nx, Ny, Lx, Ly, gauss5())
    kx, ky = 2 * np.pi / Lx, 2 * np.pi / Ly
    U = make_state(1.0 + 0.04 * np.sin(kx * x) * np.cos(ky * y) + 0.01 * np.cos(2 * kx * x),
                   0.08 * np.cos(kx * x) * (1 - bc), -0.05 * np.sin(ky * y) * (1 - bc),
                   0.02 * np.sin(kx * x), 0.01 * np.cos(ky * y))
    return kw, U


def make_state(h, u, v, w, p):
    h = np.asarray(h, dtype=np.float64)
    return np.concatenate([h, h * u, h * v, h * w, h * p]).astype(np.float64)


def bump_case(bc=BC_PERIODIC, Nx=8, Ny=6, Lx=10.0, Ly=8.0):
    c = ALPHA * np.sqrt(G * 1.0)
    kw = dict(P=4, Nx=Nx, Ny=Ny, Lx=Lx, Ly=Ly, g=G, c=c, gamma=GAMMA, bc_x=bc, bc_y=bc,
              bathy_kind=BATHY_GAUSS, bathy_par=(1.0, 0.4, 0.5 * Lx, 0.5 * Ly, 6.0))
    x, y = node_coords(4, Nx, Ny, Lx, Ly, gll5())
    kx, ky = 2 * np.pi / Lx, 2 * np.pi / Ly
    H = 1.0 - 0.4 * np.exp(-((x - 0.5 * Lx) ** 2 + (y - 0.5 * Ly) ** 2) / 6.0)
    U = make_state(H + 0.04 * np.sin(kx * x) * np.cos(ky * y), 0.08 * np.cos(kx * x),
                   -0.05 * np.sin(ky * y), 0.02 * np.sin(kx * x), 0.01 * np.cos(ky * y))
    return kw, U


def lake_case(Hnod, Nd):
    z = np.zeros(Nd)
    return make_state(Hnod, z, z, z, z)


def cfg1_case():
    Nx, Ny, Lx, Ly = 128, 64, 20.0, 10.0
    kw = dict(P=4, Nx=Nx, Ny=Ny, Lx=Lx, Ly=Ly, g=G, c=ALPHA * np.sqrt(G * 1.0), gamma=GAMMA,
              bc_x=BC_PERIODIC, bc_y=BC_PERIODIC, bathy_kind=BATHY_CONST, bathy_par=(1.0,))
    x, y = node_coords(4, Nx, Ny, Lx, Ly, gll5())
    h = 1.0 + 0.05 * np.exp(-((x - 10.0) ** 2 + (y - 5.0) ** 2) / 0.5)
    z = np.zeros_like(h)
    return kw, make_state(h, z, z, z, z)


def cfg2_params(seed=2):
    """Depth profile and wave components of configuration 2."""
    H0, Hc = 0.45, 0.15
    shoal = (H0, Hc, 20.0, 10.0, 4.0, 3.0)
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.005, 0.02, 8)
    lam = rng.uniform(1.0, 4.0, 8)
    theta = rng.uniform(0.0, 2 * np.pi, 8)
    phase = rng.uniform(0.0, 2 * np.pi, 8)
    return shoal, (amp, lam, theta, phase)


def cfg2_case(Nx=2048, Ny=1024, Lx=40.0, Ly=20.0, seed=2, chunk=1 << 22):
    shoal, (amp, lam, theta, phase) = cfg2_params(seed)
    kw = dict(P=4, Nx=Nx, Ny=Ny, Lx=Lx, Ly=Ly, g=G, c=ALPHA * np.sqrt(G * shoal[0]),
              gamma=GAMMA, bc_x=BC_WALL, bc_y=BC_WALL, bathy_kind=BATHY_SHOAL,
              bathy_par=shoal)
    x, y = node_coords(4, Nx, Ny, Lx, Ly, gll5())
    Nd = x.size
    U = np.zeros(5 * Nd)
    for s in range(0, Nd, chunk):
        xs, ys = x[s:s + chunk], y[s:s + chunk]
        dx, dy = (xs - shoal[2]) / shoal[4], (ys - shoal[3]) / shoal[5]
        r2 = dx * dx + dy * dy
        q = np.clip(1.0 - r2, 0.0, None)
        H = shoal[0] - (shoal[0] - shoal[1]) * q ** 3
        eta = np.zeros_like(xs)
        for a, l, t, ph in zip(amp, lam, theta, phase):
            k = 2 * np.pi / l
            eta += a * np.sin(k * (xs * np.cos(t) + ys * np.sin(t)) + ph)
        U[s:s + xs.size] = H + eta
    return kw, U


def cfg3_bathymetry(seed=3, Lx=20.0, Ly=10.0, H0=1.0):
    """Configuration 3's lake-at-rest bathymetry: H0 minus 5 seeded Gaussian bumps of
    height 0.05-0.3, centres uniform in the domain, widths sigma in [0.5, 2]
    (BATHY_GAUSS_SUM parameters)."""
    rng = np.random.default_rng(seed)
    par = [H0, 5]
    for _ in range(5):
        par += [rng.uniform(0.05, 0.3), rng.uniform(0, Lx), rng.uniform(0, Ly),
                rng.uniform(0.5, 2.0)]
    return tuple(par)


def cfg3_lake_case():
    Nx, Ny, Lx, Ly = 128, 64, 20.0, 10.0
    kw = dict(P=4, Nx=Nx, Ny=Ny, Lx=Lx, Ly=Ly, g=G, c=ALPHA * np.sqrt(G * 1.0), gamma=GAMMA,
              bc_x=BC_PERIODIC, bc_y=BC_PERIODIC, bathy_kind=BATHY_GAUSS_SUM,
              bathy_par=cfg3_bathymetry())
    return kw


def random_case(seed):
    """A seeded random case: mesh, boundaries, g, gamma, c, Manning, solution points,
    bathymetry and a smooth random state. In a walled direction the reference (on the
    mirror-doubled domain) sees the wall problem only for bathymetry symmetric across the
    wall, so a bump there is centred on 0 or on L."""
    import oracle as O  # node coordinates and the set-up's nodal depth

    rng = np.random.default_rng(seed)
    Nx, Ny = int(rng.integers(2, 10)), int(rng.integers(2, 10))
    Lx, Ly = float(rng.uniform(0.5, 3.0) * Nx), float(rng.uniform(0.5, 3.0) * Ny)
    bc_x, bc_y = int(rng.integers(0, 2)), int(rng.integers(0, 2))
    g = float(rng.uniform(1.0, 20.0))
    kw = dict(P=4, Nx=Nx, Ny=Ny, Lx=Lx, Ly=Ly, g=g, gamma=float(rng.uniform(0.5, 3.0)),
              c=float(rng.uniform(0.0, 3.0) * np.sqrt(g)), bc_x=bc_x, bc_y=bc_y,
              nManning=0.0 if rng.random() < 0.5 else float(rng.uniform(0.005, 0.05)))
    points = O.POINTS_GAUSS if rng.random() < 0.25 else O.POINTS_GLL
    H0 = float(rng.uniform(0.5, 1.5))
    kind = O.BATHY_NONE if points == O.POINTS_GAUSS else int(rng.integers(0, 3))
    if kind == O.BATHY_CONST:
        par = (H0,)
    elif kind == O.BATHY_GAUSS:
        xc = float(rng.choice([0.0, Lx])) if bc_x else float(rng.uniform(0, Lx))
        yc = float(rng.choice([0.0, Ly])) if bc_y else float(rng.uniform(0, Ly))
        par = (H0, float(rng.uniform(0.0, 0.5) * H0), xc, yc, float(rng.uniform(0.5, 3.0) * Lx))
    else:
        par = ()
    kw.update(bathy_kind=kind, bathy_par=par, points=points)
    o = O.Oracle(**kw)
    x, y = o.node_coords()
    H = o.bathymetry()["Hnod"] if kind != O.BATHY_NONE else np.ones_like(x)
    def smooth(a):
        kx, ky = rng.integers(1, 3, 2) * 2 * np.pi / np.array([Lx, Ly])
        return a * np.sin(kx * x + rng.uniform(0, 6.3)) * np.cos(ky * y + rng.uniform(0, 6.3))
    U = o.make_state(H + smooth(0.05 * H0), smooth(0.1), smooth(0.1), smooth(0.02), smooth(0.02))
    return kw, U
