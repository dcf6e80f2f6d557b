"""Pins the CPU oracle (oracle/sgn_oracle.c) before it is trusted as the checker.

* against the reference's own CPU solver compiled from its sources (oracle/_ref),
  bit for bit: rhs on periodic and walled domains, bathymetry set-up, adaptive runs;
* against the committed golden fixtures generated from that reference
  (tests/golden/make_golden.py), so the pin holds where the reference is absent;
* against the reference's known-answer gates (test/test_sgn2d.cpp:55-179) and its published
  spatial-convergence errors (results/convergence2d.csv, P = 4).
"""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

import oracle as O
from cases import bump_case, cfg1_case, gauss_case, random_case, CFG1_STEPS, lake_case
from conftest import bits_equal


def oracle_for(kw, reference=False):
    return O.Oracle(reference=reference, **kw)


# --------------------------------------------------------------------------- reference
@pytest.mark.parametrize("bcx,bcy", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_rhs_bitwise_vs_reference(need_reference, bcx, bcy):
    kw, U = bump_case()
    kw = dict(kw, bc_x=bcx, bc_y=bcy)
    a, b = oracle_for(kw), oracle_for(kw, reference=True)
    assert bits_equal(a.rhs(U), b.rhs(U))
    ta, tb = a.tables(), b.tables()
    for k in ta:
        assert bits_equal(ta[k], tb[k]), k
    ba, bb = a.bathymetry(), b.bathymetry()
    for k in ("Hnod", "Hx", "Hy", "HfaceX", "HfaceY"):
        assert bits_equal(ba[k], bb[k]), k
    if bcx:
        assert bits_equal(ba["HfaceXEnd"], bb["HfaceXEnd"])
    if bcy:
        assert bits_equal(ba["HfaceYEnd"], bb["HfaceYEnd"])


@pytest.mark.parametrize("bc", [0, 1])
def test_rhs_manning_bitwise_vs_reference(need_reference, bc):
    """Manning friction branch (sgn_flux2d.h:135-142), n = 0.03."""
    kw, U = bump_case(bc)
    kw = dict(kw, nManning=0.03)
    a, b = oracle_for(kw), oracle_for(kw, reference=True)
    Ra = a.rhs(U)
    assert bits_equal(Ra, b.rhs(U))
    assert not bits_equal(Ra, oracle_for(dict(kw, nManning=0.0)).rhs(U))


@pytest.mark.parametrize("Nx,Ny", [(2, 2), (3, 5), (10, 6)])
def test_rhs_bitwise_vs_reference_sizes(need_reference, Nx, Ny):
    kw, U = bump_case(Nx=Nx, Ny=Ny)
    assert bits_equal(oracle_for(kw).rhs(U), oracle_for(kw, True).rhs(U))


@pytest.mark.parametrize("bc", [0, 1])
def test_integrate_bitwise_vs_reference(need_reference, bc):
    kw, U = bump_case(bc)
    a, b = oracle_for(kw), oracle_for(kw, True)
    dt0 = a.cfl_time_step(U, 0.5)
    assert dt0 == b.cfl_time_step(U, 0.5)
    ua, sa, _ = a.integrate_adaptive(U, 0.0, 0.02, dt0, atol=1e-10, rtol=1e-8)
    ub, sb, _ = b.integrate_adaptive(U, 0.0, 0.02, dt0, atol=1e-10, rtol=1e-8)
    for k in ("accepted", "rejected", "rhsEvals", "tReached", "dtLast", "maxNormLast"):
        assert sa[k] == sb[k], k
    assert bits_equal(ua, ub)


def test_steppers_bitwise_vs_reference(need_reference):
    kw, U = bump_case()
    a, b = oracle_for(kw), oracle_for(kw, True)
    assert bits_equal(a.bs3_step(U, 0.0, 1e-3), b.bs3_step(U, 0.0, 1e-3))
    assert bits_equal(a.rk4_step(U, 0.0, 1e-3), b.rk4_step(U, 0.0, 1e-3))
    assert a.mass(U) == b.mass(U) and a.energy(U) == b.energy(U)


def test_bathymetry_kinds_vs_reference(need_reference):
    kinds = [(O.BATHY_CONST, (0.7,)), (O.BATHY_SHOAL, (0.45, 0.15, 5.0, 4.0, 4.0, 3.0)),
             (O.BATHY_GAUSS_SUM, (1.0, 2, 0.2, 3.0, 2.0, 1.0, 0.1, 7.0, 5.0, 0.7)),
             (O.BATHY_CELLS, (4, 3, 10.0, 8.0) + tuple(np.linspace(0.5, 1.5, 12)))]
    for kind, par in kinds:
        kw, _ = bump_case(1)
        kw = dict(kw, bathy_kind=kind, bathy_par=par)
        ba, bb = oracle_for(kw).bathymetry(), oracle_for(kw, True).bathymetry()
        for k in ba:
            assert bits_equal(ba[k], bb[k]), (kind, k)


def test_cfg2_generator_vs_reference(need_reference):
    """Configuration 2's own generator (the benchmark's: walls, elliptic shoal on the 0.45
    plane, 8 seeded random-phase sines; sgnb.workloads) on a 256 x 128 mesh of the same
    40 x 20 basin: the restatement's rhs, cfl step and one bs3Step equal the reference's
    bit for bit. The reference sees the walls through mirror doubling; the shoal lies
    inside [16, 24] x [7, 13], so the doubled domain's depth is the walled problem's."""
    from sgnb import workloads as W

    kw = W.cfg2_solver_args(256, 128)
    U = W.cfg2_state_torch(256, 128, device="cpu").numpy()
    a, b = oracle_for(kw), oracle_for(kw, reference=True)
    R = a.rhs(U)
    assert bits_equal(R, b.rhs(U))
    assert np.abs(R).max() > 0
    dt = a.cfl_time_step(U, 0.5)
    assert dt == b.cfl_time_step(U, 0.5)
    assert bits_equal(a.bs3_step(U, 0.0, dt), b.bs3_step(U, 0.0, dt))


@pytest.mark.parametrize("seed", range(40))
def test_random_cases_vs_reference(need_reference, seed):
    """Forty seeded random cases: the restatement's rhs equals the reference's bit for bit
    (Gauss points with a wall: to round-off, see test_gauss_vs_reference), and where both
    directions are periodic one bs3Step and one rk4Step also agree bit for bit."""
    kw, U = random_case(seed)
    a, b = oracle_for(kw), oracle_for(kw, reference=True)
    R, Rref = a.rhs(U), b.rhs(U)
    if kw["points"] == O.POINTS_GAUSS and (kw["bc_x"] or kw["bc_y"]):
        assert np.abs(R - Rref).max() <= 1e-13 * np.abs(Rref).max()
    else:
        assert bits_equal(R, Rref), kw
        if not (kw["bc_x"] or kw["bc_y"]):
            dt = 0.2 * a.cfl_time_step(U, 0.5)
            assert bits_equal(a.bs3_step(U, 0.0, dt), b.bs3_step(U, 0.0, dt))
            assert bits_equal(a.rk4_step(U, 0.0, dt), b.rk4_step(U, 0.0, dt))


# --------------------------------------------------------------------------- golden
@pytest.mark.parametrize("tag,bc", [("bump", 0), ("wall", 1)])
def test_rhs_vs_golden(golden, tag, bc):
    kw, U = bump_case(bc)
    assert bits_equal(U, golden[f"{tag}_U"])
    o = oracle_for(kw)
    assert bits_equal(o.rhs(U), golden[f"{tag}_R"])
    b = o.bathymetry()
    for k in ("Hnod", "Hx", "Hy", "HfaceX", "HfaceY"):
        assert bits_equal(b[k], golden[f"{tag}_{k}"]), k


def test_adaptive_run_vs_golden(golden):
    kw, U = bump_case()
    o = oracle_for(kw)
    dt0 = o.cfl_time_step(U, 0.5)
    assert dt0 == golden["run_dt0"][0]
    u, st, _ = o.integrate_adaptive(U, 0.0, 0.05, dt0, atol=1e-10, rtol=1e-8)
    assert [st["accepted"], st["rejected"], st["rhsEvals"]] == list(golden["run_stats"])
    assert bits_equal(u, golden["run_U"])


def test_cfg1_vs_golden(golden):
    """Configuration 1: rhs checksum and the 100-accepted-step run of the reference."""
    kw, U = cfg1_case()
    o = oracle_for(kw)
    R = o.rhs(U)
    assert hashlib.sha256(R.tobytes()).hexdigest() == str(golden["cfg1_rhs_sha"][0])
    dt0 = o.cfl_time_step(U, 0.5)
    assert dt0 == golden["cfg1_dt0"][0]
    u, st, _ = o.integrate_adaptive(U, 0.0, float(golden["cfg1_tEnd"][0]), dt0)
    assert st["accepted"] == CFG1_STEPS
    assert [st["accepted"], st["rejected"], st["rhsEvals"]] == list(golden["cfg1_stats"])
    assert hashlib.sha256(u.tobytes()).hexdigest() == str(golden["cfg1_final_sha"][0])
    assert o.mass(U) == golden["cfg1_mass"][0] and o.mass(u) == golden["cfg1_mass"][1]


# --------------------------------------------------------------------------- Gauss points
def test_gauss_vs_golden(golden):
    """Gauss-Legendre points: FR tables, rhs and a short adaptive run of the reference."""
    kw, U = gauss_case()
    o = oracle_for(kw)
    for k, a in o.tables().items():
        assert bits_equal(a, golden[f"gauss_{k}"]), k
    assert bits_equal(U, golden["gauss_U"])
    assert bits_equal(o.rhs(U), golden["gauss_R"])
    u, st, _ = o.integrate_adaptive(U, 0.0, 0.05, o.cfl_time_step(U, 0.5), atol=1e-10,
                                    rtol=1e-8)
    assert [st["accepted"], st["rejected"], st["rhsEvals"]] == list(golden["gauss_run_stats"])
    assert bits_equal(u, golden["gauss_run_U"])


@pytest.mark.parametrize("bc", [0, 1])
def test_gauss_vs_reference(need_reference, bc):
    """Periodic: bit for bit. Walls: the restatement mirrors the own trace, the reference
    (on the mirror-doubled domain) interpolates the mirror element's trace with lR, which
    equals lL reversed to round-off only."""
    kw, U = gauss_case(bc, Nx=7, Ny=5)
    R, Rref = oracle_for(kw).rhs(U), oracle_for(kw, reference=True).rhs(U)
    if bc == 0:
        assert bits_equal(R, Rref)
    else:
        # round-off of the face traces (O(1) fluxes); the h field's own rhs is small here
        assert np.abs(R - Rref).max() <= 1e-13 * np.abs(Rref).max()
        assert not np.array_equal(R, oracle_for(dict(kw, bc_x=0, bc_y=0)).rhs(U))


def test_gauss_needs_flat_bottom_and_keeps_freestream():
    kw, _ = gauss_case()
    with pytest.raises(ValueError):
        oracle_for(dict(kw, bathy_kind=O.BATHY_GAUSS, bathy_par=(1.0, 0.4, 5.0, 4.0, 6.0)))
    o = oracle_for(kw)
    n = o.Nd
    U = o.make_state(np.full(n, 1.0), np.full(n, 0.5), np.full(n, -0.3), np.zeros(n), np.zeros(n))
    assert np.abs(o.rhs(U)).max() < 1e-11
    # Gauss quadrature integrates the constant depth exactly: mass = h Lx Ly
    assert abs(o.mass(U) - 80.0) < 1e-12


# --------------------------------------------------------------------------- known answers
def test_lake_at_rest():
    """test/test_sgn2d.cpp:55-66: max|RHS| < 1e-12 over the bump."""
    kw, _ = bump_case()
    o = oracle_for(kw)
    U = lake_case(o.bathymetry()["Hnod"], o.Nd)
    assert np.abs(o.rhs(U)).max() < 1e-12


def test_freestream():
    """test/test_sgn2d.cpp:68-77: constant h, u, v on a flat bottom, max|RHS| < 1e-11."""
    kw, _ = bump_case()
    o = oracle_for(dict(kw, bathy_kind=O.BATHY_NONE, bathy_par=()))
    n = o.Nd
    U = o.make_state(np.full(n, 1.0), np.full(n, 0.5), np.full(n, -0.3), np.zeros(n), np.zeros(n))
    assert np.abs(o.rhs(U)).max() < 1e-11


def test_mass_conservation():
    """test/test_sgn2d.cpp:159-179: relative mass drift < 1e-13 over an adaptive run."""
    kw, _ = bump_case()
    o = oracle_for(kw)
    x, y = o.node_coords()
    H = o.bathymetry()["Hnod"]
    z = np.zeros(o.Nd)
    U = o.make_state(H + 0.03 * np.sin(2 * np.pi * x / 10) * np.cos(2 * np.pi * y / 8), z, z, z, z)
    M0 = o.mass(U)
    u, st, _ = o.integrate_adaptive(U, 0.0, 0.1, o.cfl_time_step(U, 0.5), atol=1e-9, rtol=1e-7)
    assert st["aborted"] == 0 and np.isfinite(u).all()
    assert abs(o.mass(u) - M0) / abs(M0) < 1e-13


def _mms(x, y, t, c2, g=9.81, gamma=1.5):
    """Manufactured solution h = 1 + ah cos phi, u = au cos phi, v = av cos phi,
    w = aw sin phi, p = ap cos phi, phi = kx x + ky y - omega t on the unit square
    (the construction of the reference's apps/convergence2d.cpp), and the forcing
    d_t U - R_cont(U) of the continuous 2D system."""
    ah, au, av, aw, ap = 0.10, 0.15, 0.12, 0.05, 0.03
    kx = ky = 2 * np.pi
    om = 1.0
    ph = kx * x + ky * y - om * t
    C, S = np.cos(ph), np.sin(ph)
    h, u, v, w, p = 1 + ah * C, au * C, av * C, aw * S, ap * C
    d = lambda a, k: -a * k * S  # derivative of a cos(phi) along a direction of wavenumber k
    hx, ux, vx, px = d(ah, kx), d(au, kx), d(av, kx), d(ap, kx)
    hy, uy, vy, py = d(ah, ky), d(au, ky), d(av, ky), d(ap, ky)
    wx, wy = aw * kx * C, aw * ky * C
    ht, ut, vt, pt = ah * om * S, au * om * S, av * om * S, ap * om * S
    wt = -aw * om * C
    dt = [ht, ht * u + h * ut, ht * v + h * vt, ht * w + h * wt, ht * p + h * pt]
    fx = [hx * u + h * ux,
          hx * u * u + 2 * h * u * ux + g * h * hx + hx * p + h * px,
          hx * u * v + h * ux * v + h * u * vx,
          hx * u * w + h * ux * w + h * u * wx,
          (hx * u + h * ux) * (p + c2) + h * u * px]
    gy = [hy * v + h * vy,
          hy * u * v + h * uy * v + h * u * vy,
          hy * v * v + 2 * h * v * vy + g * h * hy + hy * p + h * py,
          hy * v * w + h * vy * w + h * v * wy,
          (hy * v + h * vy) * (p + c2) + h * v * py]
    src = [0, 0, 0, gamma * p, c2 * u * hx + c2 * v * hy - 2 * c2 * w]
    forcing = np.concatenate([dt[k] + fx[k] + gy[k] - src[k] for k in range(5)])
    return (h, u, v, w, p), forcing


@pytest.mark.parametrize("N,expected", [(4, 1.326890e-05), (8, 8.534216e-07), (16, 5.307817e-08)])
def test_mms_convergence_known_answer(N, expected):
    """Spatial error of h for P = 4 against the reference's published table
    (results/convergence2d.csv: 1.326890e-05, 8.534216e-07, 5.307817e-08), RK4 with
    dt = 0.15 dx_eff / sqrt(1.2 g + c^2) to t = 0.1."""
    g, c = 9.81, 3.0 * np.sqrt(9.81)
    c2 = c * c
    o = O.Oracle(P=4, Nx=N, Ny=N, Lx=1.0, Ly=1.0, g=g, c=c, gamma=1.5)
    x, y = o.node_coords()
    prim, _ = _mms(x, y, 0.0, c2)
    U = o.make_state(*prim)
    dxeff = (1.0 / N) / 9.0
    dt = 0.15 * dxeff / np.sqrt(g * 1.2 + c2)
    nstep = int(np.ceil(0.1 / dt))
    dt = 0.1 / nstep
    f = lambda t, u: o.rhs(u) + _mms(x, y, t, c2)[1]
    t = 0.0
    for _ in range(nstep):
        k1 = f(t, U)
        k2 = f(t + 0.5 * dt, U + 0.5 * dt * k1)
        k3 = f(t + 0.5 * dt, U + 0.5 * dt * k2)
        k4 = f(t + dt, U + dt * k3)
        U = U + (dt / 6.0) * (k1 + 2 * k2 + 2 * k3 + k4)
        t += dt
    qw = o.tables()["qw"]
    w2 = np.tile(np.outer(qw, qw).reshape(-1), N * N)  # a fastest: w_a w_b
    J = (0.5 / N) ** 2
    err = np.sqrt(np.sum(w2 * J * (U[: o.Nd] - _mms(x, y, 0.1, c2)[0][0]) ** 2))
    assert err == pytest.approx(expected, rel=2e-6)


def test_cfg1_controller_sensitivity():
    """Documents a property of the reference algorithm on configuration 1: the adaptive
    controller amplifies a 1-ulp change of dt0 to > 1e-7 relative in the error norm within
    nine steps, so free adaptive runs are compared at tolerance, not bit for bit."""
    kw, U = cfg1_case()
    o = oracle_for(kw)
    dt0 = o.cfl_time_step(U, 0.5)
    _, _, l1 = o.integrate_adaptive(U, 0.0, 1e9, dt0, max_log=16, stop_after=10)
    _, _, l2 = o.integrate_adaptive(U, 0.0, 1e9, np.nextafter(dt0, 1.0), max_log=16,
                                    stop_after=10)
    rel = np.abs(l1[:10, 2] - l2[:10, 2]) / l1[:10, 2]
    assert rel[0] < 1e-12 and rel[9] > 1e-7
