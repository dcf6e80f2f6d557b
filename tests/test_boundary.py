"""The C-ABI boundary without a GPU: the library loads, exports every entry point that
include/sgnb.h declares, validates its arguments like the reference (std::invalid_argument
there, status codes here), and its host set-up reproduces the reference's tables and
bathymetry bit for bit."""
from __future__ import annotations

import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O
import sgnb
from cases import bump_case
from conftest import ROOT, bits_equal

HEADERS = [os.path.join(ROOT, "include", "sgnb.h")]


def declared_symbols():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        names |= set(re.findall(r"\b(sgnb_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = sgnb.lib()
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", sgnb.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (sgnb_[a-z0-9_]+)", out))
    assert set(declared_symbols()) <= exported


def test_python_signatures_cover_header():
    assert set(declared_symbols()) == set(sgnb.SIGNATURES)


def test_fr_tables_bitwise():
    mine = sgnb.fr_tables(4)
    ref = O.Oracle().tables()
    for k in ref:
        assert bits_equal(mine[k], ref[k]), k


def test_gauss_tables_bitwise(golden):
    """FROperators1D(4, GaussLegendre): the reference's tables, committed as fixtures."""
    mine = sgnb.fr_tables(4, points=sgnb.POINTS_GAUSS)
    for k in ("nodes", "D", "lL", "lR", "gLp", "gRp", "qw"):
        assert bits_equal(mine[k], golden[f"gauss_{k}"]), k
    with pytest.raises(sgnb.SgnbError) as ei:
        sgnb.fr_tables(4, points=3)
    assert ei.value.status == 1


def test_gauss_points_need_a_flat_bottom():
    """SGN2D refuses bathymetry with non-GLL points (sgn2d.cpp:46-47): SGNB_ERR_INVALID,
    before any device is touched; the flat bottom sets up all-zero statics."""
    with pytest.raises(sgnb.SgnbError) as ei:
        sgnb.SGN2DB200(Nx=8, Ny=6, points=sgnb.POINTS_GAUSS, bathy_kind=sgnb.BATHY_CONST,
                       bathy_par=(1.0,))
    assert ei.value.status == 1
    with pytest.raises(sgnb.SgnbError) as ei:
        sgnb.SGN2DB200(Nx=8, Ny=6, points=sgnb.POINTS_GAUSS, precision=sgnb.MIXED)
    assert ei.value.status == 2
    h = sgnb._DescHolder(4, 8, 6, 10.0, 8.0, 9.81, 0.0, 1.5, 0.0, 0, 0, sgnb.FP64_EXACT, 0,
                         sgnb.BATHY_NONE, (), None, None, sgnb.POINTS_GAUSS)
    import ctypes as C

    out = [np.ones(n) for n in (1200, 1200, 1200, 240, 240, 30, 40)]
    assert sgnb.lib().sgnb_setup_bathymetry(C.byref(h.desc), *(sgnb._ptr(a) for a in out)) == 0
    assert all(not a.any() for a in out)


KINDS = [
    (O.BATHY_NONE, ()),
    (O.BATHY_CONST, (1.0,)),
    (O.BATHY_GAUSS, (1.0, 0.4, 5.0, 4.0, 6.0)),
    (O.BATHY_SHOAL, (0.45, 0.15, 5.0, 4.0, 4.0, 3.0)),
    (O.BATHY_GAUSS_SUM, (1.0, 2, 0.2, 3.0, 2.0, 1.0, 0.1, 7.0, 5.0, 0.7)),
    (O.BATHY_CELLS, (4, 3, 10.0, 8.0) + tuple(np.linspace(0.5, 1.5, 12))),
]


@pytest.mark.parametrize("kind,par", KINDS)
@pytest.mark.parametrize("bc", [0, 1])
def test_host_bathymetry_bitwise(kind, par, bc):
    mine = sgnb.setup_bathymetry(Nx=8, Ny=6, Lx=10.0, Ly=8.0, bathy_kind=kind, bathy_par=par,
                                 bc_x=bc, bc_y=bc)
    ref = O.Oracle(Nx=8, Ny=6, Lx=10.0, Ly=8.0, bc_x=bc, bc_y=bc, bathy_kind=kind,
                   bathy_par=par).bathymetry()
    for k in ref:
        assert bits_equal(mine[k], ref[k]), k


@pytest.mark.parametrize("kw,code", [
    (dict(P=3), 2),             # only P = 4 is built
    (dict(Nx=1), 1),            # SGN2D: Nx, Ny >= 2 (src/solver/sgn2d.cpp:36)
    (dict(nManning=-0.02), 1),  # Manning coefficient must be >= 0
    (dict(bc_x=7), 1),
    (dict(precision=9), 2),
    (dict(bathy_kind=42), 1),
    (dict(bathy_kind=sgnb.BATHY_GAUSS, bathy_par=(1.0,)), 1),  # parameter vector too short
    (dict(Ny=1), 1),            # SGN2D: Nx, Ny >= 2
    (dict(Lx=0.0), 1),          # a degenerate domain (hx = Lx / Nx, mesh2d.h:27) is refused
    (dict(Ly=-1.0), 1),
    (dict(Nx=9269, Ny=9268), 1),  # 25 Nx Ny nodes per field must stay below 2^31
])
def test_create_rejects_bad_arguments(kw, code):
    args = dict(Nx=8, Ny=6)
    args.update(kw)
    with pytest.raises(sgnb.SgnbError) as ei:
        sgnb.SGN2DB200(**args)
    assert ei.value.status == code


def test_largest_mesh_passes_validation():
    """9268 x 9268 elements (25 Nx Ny = 2,147,395,600 nodes per field, just below 2^31) passes
    argument validation and reaches the device check; one element column more is refused
    above."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is visible (the mesh would be allocated)")
    with pytest.raises(sgnb.SgnbError) as ei:
        sgnb.SGN2DB200(Nx=9268, Ny=9268)
    assert ei.value.status == 8


def test_create_without_device_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is visible")
    with pytest.raises(sgnb.SgnbError) as ei:
        sgnb.SGN2DB200(Nx=8, Ny=6)
    assert ei.value.status == 8  # SGNB_ERR_NO_DEVICE: no CPU fallback


def test_cases_match_oracle_coordinates():
    kw, _ = bump_case()
    o = O.Oracle(**kw)
    from cases import node_coords, gll5

    x, y = node_coords(4, kw["Nx"], kw["Ny"], kw["Lx"], kw["Ly"], gll5())
    xo, yo = o.node_coords()
    assert np.abs(x - xo).max() < 1e-14 and np.abs(y - yo).max() < 1e-14


def test_host_buffers_must_be_contiguous_float64():
    """Every host array handed to the library goes through sgnb._ptr, which refuses other
    dtypes and strided views (the library reads and writes plain double arrays)."""
    import numpy as np

    assert sgnb._ptr(None) is None
    sgnb._ptr(np.zeros(4))
    with pytest.raises(ValueError):
        sgnb._ptr(np.zeros(4, dtype=np.float32))
    with pytest.raises(ValueError):
        sgnb._ptr(np.zeros(8)[::2])
