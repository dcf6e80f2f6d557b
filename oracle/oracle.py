"""ctypes front-end for the CPU oracle libraries (test infrastructure only).

The oracle is the checker for the CUDA path: tests, the smoke check and the CPU
baseline of bench.py load it; product code never does. Two libraries share the C
interface of sgn_oracle.h:

* ``liboracle.so`` -- the plain-C restatement of the reference algorithm
  (sgn_oracle.c);
* ``_ref/libsgnref.so`` -- the reference's own CPU sources compiled from where they
  lie by ``make ref`` (present only where the reference tree was available at build
  time; it travels with the repository snapshot as a built file).

``Oracle`` mirrors the reference class ``sgn::SGN2D`` (src/solver/sgn2d.h:49-113) and
the integrators of src/solver/rk.h, operating on numpy arrays in the reference's
variable-major layout ``U[v*Nd + e*25 + a + 5*b]``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_RESTATEMENT = os.path.join(HERE, "liboracle.so")
LIB_REFERENCE = os.path.join(HERE, "_ref", "libsgnref.so")

BC_PERIODIC = 0
BC_WALL = 1
POINTS_GLL = 0    # solution points (PointSet, src/core/fr_operators.h:51)
POINTS_GAUSS = 1

BATHY_NONE = 0
BATHY_CONST = 1
BATHY_GAUSS = 2
BATHY_SHOAL = 3
BATHY_GAUSS_SUM = 4
BATHY_CELLS = 5

# AdaptiveRKOptions defaults (src/solver/rk.h:53-61)
DEFAULT_OPTS = dict(atol=1e-8, rtol=1e-6, dtMin=1e-13, dtMax=1e30, safety=0.9,
                    facMin=0.2, facMax=5.0)

_libs: dict[str, C.CDLL] = {}
_dp = C.POINTER(C.c_double)


def reference_dir() -> str:
    """The reference project's source tree: SGN_REFERENCE_DIR, else the checkout beside
    this repository (the directory holding the repository's own directory)."""
    return os.environ.get("SGN_REFERENCE_DIR",
                          os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))


def build() -> None:
    """Compile liboracle.so (and _ref/libsgnref.so when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    ref = reference_dir()
    if os.path.isdir(os.path.join(ref, "src", "solver")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref}"], check=True)


def reference_rhs_1d(P, N, L, g, c, gamma, U1):
    """The reference's 1D solver's right-hand side (flat bottom, periodic), var-major
    (h, hu, hw, hp); needs the compiled reference."""
    lib = _load(LIB_REFERENCE)
    U1 = np.ascontiguousarray(U1, dtype=np.float64)
    out = np.empty_like(U1)
    lib.or_rhs_1d(P, N, L, g, c, gamma, _ptr(U1), _ptr(out))
    return out


def reference_available() -> bool:
    return os.path.exists(LIB_REFERENCE)


def _load(path: str) -> C.CDLL:
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        if path == LIB_RESTATEMENT:
            build()
        else:
            raise FileNotFoundError(path)
    lib = C.CDLL(path)
    lib.or_create.restype = C.c_void_p
    lib.or_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                              C.c_double, C.c_double, C.c_double, C.c_double,
                              C.c_int, C.c_int, C.c_int, _dp, C.c_int]
    lib.or_create_points.restype = C.c_void_p
    lib.or_create_points.argtypes = lib.or_create.argtypes + [C.c_int]
    lib.or_destroy.argtypes = [C.c_void_p]
    lib.or_ndof.restype = C.c_long
    lib.or_ndof.argtypes = [C.c_void_p]
    lib.or_tables.argtypes = [C.c_void_p] + [_dp] * 7
    lib.or_bathymetry.argtypes = [C.c_void_p] + [_dp] * 7
    if hasattr(lib, "or_rhs_1d"):
        lib.or_rhs_1d.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                  C.c_double, _dp, _dp]
        lib.or_rhs_1d.restype = C.c_int
    if hasattr(lib, "or_write_vtk"):
        lib.or_write_vtk.argtypes = [C.c_void_p, _dp, C.c_char_p]
        lib.or_write_vtk.restype = C.c_int
    if hasattr(lib, "or_set_bathymetry"):
        lib.or_set_bathymetry.argtypes = [C.c_void_p] + [_dp] * 7
    lib.or_node_coords.argtypes = [C.c_void_p, _dp, _dp]
    lib.or_rhs.argtypes = [C.c_void_p, _dp, _dp]
    lib.or_rhs.restype = C.c_int
    for name in ("or_max_wave_speed", "or_mass", "or_energy"):
        getattr(lib, name).restype = C.c_double
        getattr(lib, name).argtypes = [C.c_void_p, _dp]
    lib.or_cfl_time_step.restype = C.c_double
    lib.or_cfl_time_step.argtypes = [C.c_void_p, _dp, C.c_double]
    lib.or_rk4_step.argtypes = [C.c_void_p, C.c_double, C.c_double, _dp]
    lib.or_bs3_step.argtypes = [C.c_void_p, C.c_double, C.c_double, _dp]
    lib.or_integrate_adaptive.restype = C.c_long
    lib.or_integrate_adaptive.argtypes = [C.c_void_p, _dp, C.c_double, C.c_double,
                                          C.c_double, _dp, _dp, _dp, C.c_long]
    _libs[path] = lib
    return lib


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


class Oracle:
    """CPU solver with the interface of sgn::SGN2D plus the rk.h integrators."""

    def __init__(self, P=4, Nx=8, Ny=6, Lx=10.0, Ly=8.0, g=9.81, c=0.0, gamma=1.5,
                 nManning=0.0, bc_x=BC_PERIODIC, bc_y=BC_PERIODIC, bathy_kind=BATHY_NONE,
                 bathy_par=(), reference=False, points=POINTS_GLL):
        self.lib = _load(LIB_REFERENCE if reference else LIB_RESTATEMENT)
        self.P, self.Nx, self.Ny, self.Lx, self.Ly = P, Nx, Ny, Lx, Ly
        self.np_ = P + 1
        self.bc_x, self.bc_y = bc_x, bc_y
        self._bp = np.ascontiguousarray(np.asarray(bathy_par, dtype=np.float64).reshape(-1))
        if self._bp.size == 0:
            self._bp = np.zeros(1)
        self.points = points
        self.h = self.lib.or_create_points(P, Nx, Ny, Lx, Ly, g, c, gamma, nManning, bc_x,
                                           bc_y, bathy_kind, _ptr(self._bp),
                                           int(self._bp.size), points)
        if not self.h:
            raise ValueError("invalid solver arguments")
        self.Nd = int(self.lib.or_ndof(self.h))
        self.n = 5 * self.Nd

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.or_destroy(self.h)
            self.h = None

    # --- set-up accessors --------------------------------------------------
    def tables(self):
        n = self.np_
        out = {k: np.zeros(n) for k in ("nodes", "lL", "lR", "gLp", "gRp", "qw")}
        out["D"] = np.zeros(n * n)
        self.lib.or_tables(self.h, _ptr(out["nodes"]), _ptr(out["D"]), _ptr(out["lL"]),
                           _ptr(out["lR"]), _ptr(out["gLp"]), _ptr(out["gRp"]),
                           _ptr(out["qw"]))
        return out

    def bathymetry(self):
        nf = self.Nx * self.Ny * self.np_
        out = dict(Hnod=np.zeros(self.Nd), Hx=np.zeros(self.Nd), Hy=np.zeros(self.Nd),
                   HfaceX=np.zeros(nf), HfaceY=np.zeros(nf),
                   HfaceXEnd=np.zeros(self.Ny * self.np_),
                   HfaceYEnd=np.zeros(self.Nx * self.np_))
        self.lib.or_bathymetry(self.h, *(_ptr(out[k]) for k in (
            "Hnod", "Hx", "Hy", "HfaceX", "HfaceY", "HfaceXEnd", "HfaceYEnd")))
        return out

    def write_vtk(self, U, path):
        """The reference's VTK frame writer (compiled reference only, periodic domains)."""
        if not hasattr(self.lib, "or_write_vtk"):
            raise NotImplementedError("write_vtk needs the compiled reference (reference=True)")
        U = np.ascontiguousarray(U, dtype=np.float64)
        if self.lib.or_write_vtk(self.h, _ptr(U), os.fsencode(path)) != 0:
            raise ValueError("the reference writer runs on periodic domains only")

    def set_bathymetry(self, arrays):
        """Replaces the depth statics (keys as returned by bathymetry(); missing keys keep
        the current array). Restatement only."""
        keys = ("Hnod", "Hx", "Hy", "HfaceX", "HfaceY", "HfaceXEnd", "HfaceYEnd")
        keep = [np.ascontiguousarray(arrays[k], dtype=np.float64) if k in arrays else None
                for k in keys]
        self.lib.or_set_bathymetry(self.h, *(_ptr(a) if a is not None else None for a in keep))

    def node_coords(self):
        x, y = np.zeros(self.Nd), np.zeros(self.Nd)
        self.lib.or_node_coords(self.h, _ptr(x), _ptr(y))
        return x, y

    def make_state(self, h, u, v, w, p):
        """SGN2D::makeState (sgn2d.cpp:107-120): primitives -> conserved, var-major."""
        h = np.asarray(h, dtype=np.float64)
        return np.concatenate([h, h * u, h * v, h * w, h * p]).astype(np.float64)

    # --- operators -----------------------------------------------------------
    def rhs(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.size == self.n
        dU = np.empty(self.n)
        self.lib.or_rhs(self.h, _ptr(U), _ptr(dU))
        return dU

    def max_wave_speed(self, U):
        return self.lib.or_max_wave_speed(self.h, _ptr(np.ascontiguousarray(U)))

    def cfl_time_step(self, U, cfl):
        return self.lib.or_cfl_time_step(self.h, _ptr(np.ascontiguousarray(U)), cfl)

    def mass(self, U):
        return self.lib.or_mass(self.h, _ptr(np.ascontiguousarray(U)))

    def energy(self, U):
        return self.lib.or_energy(self.h, _ptr(np.ascontiguousarray(U)))

    def rk4_step(self, U, t, dt):
        u = np.array(U, dtype=np.float64, copy=True)
        self.lib.or_rk4_step(self.h, t, dt, _ptr(u))
        return u

    def bs3_step(self, U, t, dt):
        u = np.array(U, dtype=np.float64, copy=True)
        self.lib.or_bs3_step(self.h, t, dt, _ptr(u))
        return u

    def integrate_adaptive(self, U, t0, tEnd, dt0, max_log=0, stop_after=0, **opts):
        """integrateAdaptive (src/solver/rk.cpp:67-164). stop_after > 0 ends the run after
        that many accepted steps (restatement only); max_log > 0 returns the attempt log
        rows (t, dt, errNorm, accepted)."""
        o = dict(DEFAULT_OPTS)
        o.update(opts)
        ov = np.array([o[k] for k in ("atol", "rtol", "dtMin", "dtMax", "safety",
                                      "facMin", "facMax")] + [float(stop_after)],
                      dtype=np.float64)
        u = np.array(U, dtype=np.float64, copy=True)
        stats = np.zeros(7)
        log = np.zeros(4 * max(max_log, 1))
        na = self.lib.or_integrate_adaptive(self.h, _ptr(u), t0, tEnd, dt0, _ptr(ov),
                                            _ptr(stats), _ptr(log) if max_log else None,
                                            max_log)
        st = dict(accepted=int(stats[0]), rejected=int(stats[1]), rhsEvals=int(stats[2]),
                  tReached=stats[3], dtLast=stats[4], maxNormLast=stats[5],
                  aborted=int(stats[6]), attempts=int(na))
        attempts = log[: 4 * min(na, max_log)].reshape(-1, 4) if max_log else None
        return u, st, attempts
