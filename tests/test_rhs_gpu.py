"""Right-hand side on the B200 through the C ABI, against the CPU oracle.

Exact mode (SGNB_FP64_EXACT) must be bit-identical to the oracle, which is itself bit-identical
to the reference's CPU solver (tests/test_oracle.py). Fast mode (SGNB_FP64_FAST) must agree
within 1e-13 relative per field (each field's error normalised by its largest magnitude).
The reference's own GPU gate is 1e-12 (test/test_cuda_sgn2d.cu:66-80).
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
import sgnb
from cases import bump_case, cfg1_case, lake_case
from conftest import bits_equal, rel_per_field

pytestmark = pytest.mark.gpu

FAST_TOL = 1e-13


def device(kw, precision, **extra):
    args = dict(kw)
    args.update(extra)
    return sgnb.SGN2DB200(precision=precision, **args)


@pytest.mark.parametrize("bcx,bcy", [(0, 0), (1, 1), (1, 0), (0, 1)])
def test_bump_exact_bitwise_and_fast(bcx, bcy):
    kw, U = bump_case()
    kw = dict(kw, bc_x=bcx, bc_y=bcy)
    R = O.Oracle(**kw).rhs(U)
    with device(kw, sgnb.FP64_EXACT) as d:
        assert bits_equal(d.rhs(U), R)
        d.upload(U)
        assert bits_equal(d.rhs_once(), R)
        assert bits_equal(d.download(), U)
    with device(kw, sgnb.FP64_FAST) as d:
        assert rel_per_field(d.rhs(U), R) < FAST_TOL


@pytest.mark.parametrize("bc", [0, 1])
def test_manning_friction(bc):
    """Manning friction (n = 0.03): the exact mode matches the oracle to the last-bit
    rounding of cbrt (the device's and the host's cube roots may round differently), the
    fast mode within 1e-13, the mixed mode within its FP32 tolerance."""
    kw, U = bump_case(bc)
    kw = dict(kw, nManning=0.03)
    R = O.Oracle(**kw).rhs(U)
    assert not bits_equal(R, O.Oracle(**dict(kw, nManning=0.0)).rhs(U))
    with device(kw, sgnb.FP64_EXACT) as d:
        assert rel_per_field(d.rhs(U), R) < 1e-15
    with device(kw, sgnb.FP64_FAST) as d:
        assert rel_per_field(d.rhs(U), R) < FAST_TOL
    with device(kw, sgnb.MIXED) as d:
        assert rel_per_field(d.rhs(U), R) < 2e-5


def test_golden_fixture_bitwise(golden):
    """The reference's own rhs of its GPU-parity case, from the committed fixture."""
    for tag, bc in (("bump", 0), ("wall", 1)):
        kw, U = bump_case(bc)
        with device(kw, sgnb.FP64_EXACT) as d:
            assert bits_equal(d.rhs(golden[f"{tag}_U"]), golden[f"{tag}_R"])


def test_reference_arrays_path(golden):
    """Tables and bathymetry passed in as arrays (the SGN2D accessors), as a reference
    caller building the device object from a host SGN2D would do."""
    kw, U = bump_case()
    tables = O.Oracle(**kw).tables()
    arrays = {k: golden[f"bump_{k}"] for k in ("Hnod", "Hx", "Hy", "HfaceX", "HfaceY")}
    with sgnb.SGN2DB200(P=4, Nx=kw["Nx"], Ny=kw["Ny"], Lx=kw["Lx"], Ly=kw["Ly"], c=kw["c"],
                        precision=sgnb.FP64_EXACT, tables=tables, bathy_arrays=arrays) as d:
        assert bits_equal(d.rhs(U), golden["bump_R"])


@pytest.mark.parametrize("Nx,Ny,bc", [(2, 2, 0), (2, 2, 1), (3, 2, 0), (9, 5, 1), (10, 6, 0),
                                      (17, 9, 1), (33, 7, 0), (16, 8, 1)])
def test_partial_tiles_and_wraps(Nx, Ny, bc):
    """Meshes that exercise every tile edge, periodic self-wrap (Nx = 2) and walls."""
    kw, U = bump_case(bc, Nx=Nx, Ny=Ny)
    R = O.Oracle(**kw).rhs(U)
    with device(kw, sgnb.FP64_EXACT) as d:
        assert bits_equal(d.rhs(U), R)
    with device(kw, sgnb.FP64_FAST) as d:
        assert rel_per_field(d.rhs(U), R) < FAST_TOL


def test_cfg1_rhs_checksum(golden):
    import hashlib

    kw, U = cfg1_case()
    with device(kw, sgnb.FP64_EXACT) as d:
        R = d.rhs(U)
    assert hashlib.sha256(R.tobytes()).hexdigest() == str(golden["cfg1_rhs_sha"][0])
    with device(kw, sgnb.FP64_FAST) as d:
        Rf = d.rhs(U)
    idx = golden["cfg1_idx"]
    assert rel_per_field(Rf, R) < FAST_TOL
    assert np.array_equal(R[idx], golden["cfg1_rhs_samples"])


def test_mid_run_state():
    """A state after some steps (non-trivial velocities, w and p) on walls."""
    kw, U = bump_case(1, Nx=12, Ny=10)
    o = O.Oracle(**kw)
    dt0 = o.cfl_time_step(U, 0.5)
    u, _, _ = o.integrate_adaptive(U, 0.0, 20 * dt0, dt0)
    R = o.rhs(u)
    with device(kw, sgnb.FP64_EXACT) as d:
        assert bits_equal(d.rhs(u), R)
    with device(kw, sgnb.FP64_FAST) as d:
        assert rel_per_field(d.rhs(u), R) < FAST_TOL


@pytest.mark.parametrize("prec", [sgnb.FP64_EXACT, sgnb.FP64_FAST])
def test_lake_at_rest(prec):
    """Well-balancing on the device (test/test_cuda_sgn2d.cu:82-94): max|RHS| < 1e-12."""
    kw, _ = bump_case(1)
    o = O.Oracle(**kw)
    U = lake_case(o.bathymetry()["Hnod"], o.Nd)
    with device(kw, prec) as d:
        assert np.abs(d.rhs(U)).max() < 1e-12


def test_diagnostics():
    kw, U = bump_case()
    o = O.Oracle(**kw)
    with device(kw, sgnb.FP64_EXACT) as d:
        d.upload(U)
        assert d.max_wave_speed() == o.max_wave_speed(U)
        assert d.cfl_time_step(0.5) == o.cfl_time_step(U, 0.5)
        assert d.mass() == pytest.approx(o.mass(U), rel=1e-14)
        assert d.energy() == pytest.approx(o.energy(U), rel=1e-13)
        x, y = d.node_coords()
        xo, yo = o.node_coords()
        assert bits_equal(x, xo) and bits_equal(y, yo)


def test_rhs_device_pointers_on_torch_stream():
    import torch

    kw, U = bump_case()
    R = O.Oracle(**kw).rhs(U)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s), device(kw, sgnb.FP64_EXACT) as d:
        Ut = torch.from_numpy(U).cuda()
        dUt = torch.empty_like(Ut)
        d.rhs_device(Ut.data_ptr(), dUt.data_ptr(), s.cuda_stream)
        s.synchronize()
        assert bits_equal(dUt.cpu().numpy(), R)


def test_translation_equivariance_full_size():
    """Size-independent property at the full configuration-2 mesh (2048 x 1024, periodic,
    flat depth): shifting the state by whole elements shifts the rhs bit for bit."""
    import torch

    Nx, Ny = 2048, 1024
    kw = dict(P=4, Nx=Nx, Ny=Ny, Lx=40.0, Ly=20.0, c=3.0 * np.sqrt(9.81 * 0.45),
              bathy_kind=sgnb.BATHY_CONST, bathy_par=(0.45,))
    Nd = 25 * Nx * Ny
    g = torch.Generator(device="cuda").manual_seed(0)
    U = torch.zeros(5, Ny, Nx, 25, dtype=torch.float64, device="cuda")
    U[0] = 0.45 + 0.01 * torch.rand(Ny, Nx, 25, generator=g, device="cuda", dtype=torch.float64)
    U[1:3] = 0.01 * torch.randn(2, Ny, Nx, 25, generator=g, device="cuda", dtype=torch.float64)
    U[3:] = 0.001 * torch.randn(2, Ny, Nx, 25, generator=g, device="cuda", dtype=torch.float64)
    Us = torch.roll(U, shifts=(3, 5), dims=(1, 2)).contiguous()
    for prec in (sgnb.FP64_EXACT, sgnb.FP64_FAST):
        with device(kw, prec) as d:
            R = torch.empty_like(U)
            Rs = torch.empty_like(U)
            s = torch.cuda.current_stream()
            d.rhs_device(U.data_ptr(), R.data_ptr(), s.cuda_stream)
            d.rhs_device(Us.data_ptr(), Rs.data_ptr(), s.cuda_stream)
            torch.cuda.synchronize()
            assert torch.equal(torch.roll(R, shifts=(3, 5), dims=(1, 2)), Rs)
            assert torch.isfinite(R).all()
    assert Nd == U[0].numel()


@pytest.mark.parametrize("axis", ["x", "y"])
@pytest.mark.parametrize("prec", [sgnb.FP64_EXACT, sgnb.FP64_FAST])
def test_embedding_vs_reference_1d(need_reference, axis, prec):
    """The 2D <-> 1D embedding gates of the reference (test/test_sgn2d.cpp:79-157): an x-
    (or y-) invariant state over a flat bottom, with the transverse velocity zero, gives on
    every line the reference 1D solver's right-hand side (within 1e-12, the reference's
    gate) and a zero transverse-momentum right-hand side."""
    from cases import G, gll5, make_state, node_coords

    P, Nx, Ny, Lx, Ly, H0 = 4, 8, 6, 10.0, 8.0, 1.0
    c = 3.0 * np.sqrt(G * H0)
    x, y = node_coords(P, Nx, Ny, Lx, Ly, gll5())
    s, L = (x, Lx) if axis == "x" else (y, Ly)
    k = 2 * np.pi / L
    h = H0 + 0.08 * np.sin(k * s)
    un = 0.15 * np.cos(k * s)
    z = np.zeros_like(s)
    U2 = make_state(h, un, z, 0.04 * np.sin(k * s), 0.02 * np.cos(k * s)) if axis == "x" else \
        make_state(h, z, un, 0.04 * np.sin(k * s), 0.02 * np.cos(k * s))
    with sgnb.SGN2DB200(P=P, Nx=Nx, Ny=Ny, Lx=Lx, Ly=Ly, c=c, precision=prec) as d:
        R2 = d.rhs(U2).reshape(5, Ny, Nx, 5, 5)  # [v, ey, ex, b, a]
    nd, td = (1, 2) if axis == "x" else (2, 1)
    # the 1D state: the 2D state along the line ey = 0, b = 0 (x) or ex = 0, a = 0 (y)
    U2r = U2.reshape(5, Ny, Nx, 5, 5)
    line = (lambda A: A[:, 0, :, 0, :].reshape(A.shape[0], -1)) if axis == "x" else \
        (lambda A: A[:, :, 0, :, 0].reshape(A.shape[0], -1))
    N = Nx if axis == "x" else Ny
    U1 = np.concatenate([line(U2r)[v] for v in (0, nd, 3, 4)])
    R1 = O.reference_rhs_1d(P, N, L, G, c, 1.5, U1).reshape(4, -1)
    R2l = line(R2)
    err = max(np.abs(R2l[v2] - R1[v1]).max() for v1, v2 in enumerate((0, nd, 3, 4)))
    assert err < 1e-12, err
    assert np.abs(R2[td]).max() < 1e-12
    # every line is the same line
    lines = R2[(0, nd, 3, 4), :, :, 0, :] if axis == "x" else R2[(0, nd, 3, 4), :, :, :, 0]
    assert np.abs(lines - lines[:, :1] if axis == "x" else lines - lines[:, :, :1]).max() < 1e-12


def test_host_buffer_sizes_checked():
    """Host arrays of the wrong size are refused before the library touches them."""
    kw, U = bump_case(0)
    with device(kw, sgnb.FP64_FAST) as d:
        d.upload(U)
        with pytest.raises(ValueError):
            d.upload(U[:-1])
        with pytest.raises(ValueError):
            d.download(np.empty(U.size - 1))
        with pytest.raises(ValueError):
            d.download(np.empty(U.size, dtype=np.float32))
        with pytest.raises(ValueError):
            d.rhs(U[:-1])
        with pytest.raises(ValueError):
            d.rhs_vjp(U, U[:-5])
        out = np.empty(U.size)
        assert d.download(out) is out and bits_equal(out, U)
