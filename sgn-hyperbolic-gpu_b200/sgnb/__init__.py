"""Python front-end of libsgnb.so, the B200 hyperbolic-SGN FR right-hand side and
Bogacki-Shampine 3(2) loop.

The classes mirror the reference's C++ interface (gsalanglada/sgn-hyperbolic-gpu) so that
its callers, and tests written in its style, translate line for line:

* ``SGN2DB200`` -- the device solver, with the members of ``sgn::SGN2DCuda``
  (src/cuda/sgn2d_cuda.h:30-79: ``upload``, ``download``, ``rhs_once``,
  ``integrate_adaptive``) plus the stateless ``rhs`` of ``sgn::SGN2D``
  (src/solver/sgn2d.h:78), ``node_coords``, ``make_state``, ``cfl_time_step``,
  ``mass`` and ``energy`` (sgn2d.h:70-90), and ``bs3_steps`` for a frozen-dt replay of
  ``bs3Step`` (src/solver/rk.h:50).
* ``AdaptiveRKOptions`` / ``AdaptiveRKStats`` -- src/solver/rk.h:53-72.

Every call goes through the C ABI of include/sgnb.h; there is no CPU fallback. If the
shared library is missing or no CUDA device is visible, construction raises.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# SGNB_LIBRARY=checked selects the range-checked build libsgnb_checked.so (tests)
LIB_PATH = os.path.join(HERE, "libsgnb_checked.so" if os.environ.get("SGNB_LIBRARY") == "checked"
                        else "libsgnb.so")

BC_PERIODIC = 0
BC_WALL = 1
POINTS_GLL = 0    # solution points (PointSet, src/core/fr_operators.h:51)
POINTS_GAUSS = 1  # Gauss-Legendre: flat bottom only (BATHY_NONE), FP64 modes
FP64_EXACT = 0
FP64_FAST = 1
MIXED = 2

BATHY_NONE = 0
BATHY_CONST = 1
BATHY_GAUSS = 2
BATHY_SHOAL = 3
BATHY_GAUSS_SUM = 4
BATHY_CELLS = 5
BATHY_ARRAYS = 100

STATUS = {0: "ok", 1: "invalid argument", 2: "unsupported configuration", 3: "CUDA error",
          4: "non-finite state", 5: "step size below dtMin", 6: "device wait timed out",
          7: "out of device memory", 8: "no CUDA device"}

_dp = C.POINTER(C.c_double)
_CUDA_STREAM_LEGACY = 0x1  # cudaStreamLegacy


class SgnbError(RuntimeError):
    """A non-zero sgnb_status, with the library's message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"sgnb status {status} ({STATUS.get(status, '?')}): {message}")
        self.status = status


class _Desc(C.Structure):
    _fields_ = [("P", C.c_int), ("Nx", C.c_int), ("Ny", C.c_int),
                ("Lx", C.c_double), ("Ly", C.c_double),
                ("g", C.c_double), ("c", C.c_double), ("gamma", C.c_double),
                ("nManning", C.c_double),
                ("bc_x", C.c_int), ("bc_y", C.c_int), ("precision", C.c_int), ("device", C.c_int),
                ("nodes", _dp), ("D", _dp), ("lL", _dp), ("lR", _dp), ("gLp", _dp),
                ("gRp", _dp), ("qw", _dp),
                ("bathy_kind", C.c_int), ("bathy_par", _dp), ("n_bathy_par", C.c_int),
                ("Hnod", _dp), ("Hx", _dp), ("Hy", _dp), ("HfaceX", _dp), ("HfaceY", _dp),
                ("HfaceXEnd", _dp), ("HfaceYEnd", _dp),
                ("Nx_global", C.c_int), ("ex_offset", C.c_int), ("point_set", C.c_int)]


class _Opts(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("atol", "rtol", "dtMin", "dtMax", "safety",
                                          "facMin", "facMax")]


class _Stats(C.Structure):
    _fields_ = [("accepted", C.c_longlong), ("rejected", C.c_longlong),
                ("rhsEvals", C.c_longlong), ("attempts", C.c_longlong),
                ("tReached", C.c_double), ("dtLast", C.c_double), ("maxNormLast", C.c_double),
                ("aborted", C.c_int), ("status", C.c_int), ("kernel_launches", C.c_longlong)]


@dataclasses.dataclass
class AdaptiveRKOptions:
    """src/solver/rk.h:53-61."""
    atol: float = 1e-8
    rtol: float = 1e-6
    dtMin: float = 1e-13
    dtMax: float = 1e30
    safety: float = 0.9
    facMin: float = 0.2
    facMax: float = 5.0


@dataclasses.dataclass
class AdaptiveRKStats:
    """src/solver/rk.h:64-72 plus the attempt count."""
    accepted: int = 0
    rejected: int = 0
    rhsEvals: int = 0
    attempts: int = 0
    tReached: float = 0.0
    dtLast: float = 0.0
    maxNormLast: float = 0.0
    aborted: int = 0
    kernel_launches: int = 0


_lib = None

# Every symbol include/sgnb.h declares, with its ctypes signature.
SIGNATURES = {
    "sgnb_desc_init": (None, [C.POINTER(_Desc)]),
    "sgnb_rk_opts_init": (None, [C.POINTER(_Opts)]),
    "sgnb_create": (C.c_int, [C.POINTER(_Desc), C.POINTER(C.c_void_p)]),
    "sgnb_destroy": (C.c_int, [C.c_void_p]),
    "sgnb_ndof": (C.c_longlong, [C.c_void_p]),
    "sgnb_upload": (C.c_int, [C.c_void_p, _dp]),
    "sgnb_download": (C.c_int, [C.c_void_p, _dp]),
    "sgnb_rhs_once": (C.c_int, [C.c_void_p, _dp]),
    "sgnb_rhs_host": (C.c_int, [C.c_void_p, _dp, _dp]),
    "sgnb_rhs_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sgnb_integrate_adaptive": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double,
                                          C.POINTER(_Opts), C.POINTER(_Stats)]),
    "sgnb_integrate_steps": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_longlong,
                                       C.POINTER(_Opts), C.POINTER(_Stats)]),
    "sgnb_bs3_steps": (C.c_int, [C.c_void_p, C.c_double, _dp, C.c_longlong]),
    "sgnb_rk4_steps": (C.c_int, [C.c_void_p, C.c_double, _dp, C.c_longlong]),
    "sgnb_launch_stage": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_void_p]),
    "sgnb_attempt_log": (C.c_int, [C.c_void_p, _dp, C.c_longlong, C.POINTER(C.c_longlong)]),
    "sgnb_max_wave_speed": (C.c_int, [C.c_void_p, _dp]),
    "sgnb_cfl_time_step": (C.c_int, [C.c_void_p, C.c_double, _dp]),
    "sgnb_mass": (C.c_int, [C.c_void_p, _dp]),
    "sgnb_energy": (C.c_int, [C.c_void_p, _dp]),
    "sgnb_diag_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                    C.c_double, C.c_double, C.c_double, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p]),
    "sgnb_node_coords": (C.c_int, [C.c_void_p, _dp, _dp]),
    "sgnb_state_device_ptr": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p),
                                        C.POINTER(C.c_void_p)]),
    "sgnb_fr_tables": (C.c_int, [C.c_int] + [_dp] * 7),
    "sgnb_fr_tables_points": (C.c_int, [C.c_int, C.c_int] + [_dp] * 7),
    "sgnb_setup_bathymetry": (C.c_int, [C.POINTER(_Desc)] + [_dp] * 7),
    "sgnb_fast_math": (C.c_int, [C.c_int, _dp, _dp, C.c_longlong, C.c_void_p]),
    "sgnb_checked_oob": (C.c_int, [C.c_int, C.POINTER(C.c_longlong), C.c_int]),
    "sgnb_set_ghosts": (C.c_int, [C.c_void_p, _dp, _dp]),
    "sgnb_slab_pack": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _dp, C.c_void_p]),
    "sgnb_slab_begin": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double,
                                  C.c_longlong, _dp,
                                  C.POINTER(_Opts)]),
    "sgnb_slab_launch": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "sgnb_slab_partials": (C.c_int, [C.c_void_p, C.POINTER(_dp), C.POINTER(C.c_int)]),
    "sgnb_slab_control": (C.c_int, [C.c_void_p, _dp, C.c_int, C.c_longlong, C.c_void_p]),
    "sgnb_slab_stage": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp, C.c_void_p]),
    "sgnb_enable_peer_access": (C.c_int, [C.c_int, C.c_int]),
    "sgnb_slab_control_all": (C.c_int, [C.c_void_p, C.POINTER(_dp), C.POINTER(C.c_int), C.c_int,
                                        C.c_longlong, C.c_void_p]),
    "sgnb_slab_status": (C.c_int, [C.c_void_p, C.POINTER(_Stats), C.POINTER(C.c_int),
                                   C.c_void_p]),
    "sgnb_eta_max": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double,
                               _dp, C.POINTER(C.c_longlong)]),
    "sgnb_sample_eta": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong), C.c_int, _dp]),
    "sgnb_nearest_node": (C.c_int, [C.c_void_p, C.c_double, C.c_double,
                                    C.POINTER(C.c_longlong)]),
    "sgnb_element_means": (C.c_int, [C.c_void_p, _dp]),
    "sgnb_write_vtk": (C.c_int, [C.c_void_p, C.c_char_p]),
    "sgnb_batch_create": (C.c_int, [C.POINTER(_Desc), C.c_int, C.POINTER(C.c_void_p)]),
    "sgnb_batch_destroy": (C.c_int, [C.c_void_p]),
    "sgnb_batch_size": (C.c_int, [C.c_void_p]),
    "sgnb_batch_instance": (C.c_void_p, [C.c_void_p, C.c_int]),
    "sgnb_batch_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "sgnb_batch_integrate_steps": (C.c_int, [C.c_void_p, _dp, C.c_longlong, C.POINTER(_Opts),
                                             C.POINTER(_Stats)]),
    "sgnb_batch_set_config": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "sgnb_batch_get_config": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "sgnb_batch_autotune": (C.c_int, [C.c_void_p, _dp, C.c_int, _dp]),
    "sgnb_batch_last_error": (C.c_char_p, [C.c_void_p]),
    "sgnb_adj_create": (C.c_int, [C.c_void_p, C.c_longlong, _dp, C.c_int,
                                  C.POINTER(C.c_longlong), C.c_int, C.POINTER(C.c_void_p)]),
    "sgnb_adj_destroy": (C.c_int, [C.c_void_p]),
    "sgnb_adj_forward": (C.c_int, [C.c_void_p, _dp, _dp, _dp]),
    "sgnb_adj_vjp": (C.c_int, [C.c_void_p, _dp, _dp, _dp]),
    "sgnb_rhs_vjp": (C.c_int, [C.c_void_p, _dp, _dp, _dp] + [_dp] * 7),
    "sgnb_status_string": (C.c_char_p, [C.c_int]),
    "sgnb_last_error": (C.c_char_p, [C.c_void_p]),
}


def lib() -> C.CDLL:
    """Load libsgnb.so from this package directory (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `make -C csrc` or __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a):
    if a is None:
        return None
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise ValueError("float64 C-contiguous array expected")
    return a.ctypes.data_as(_dp)


def _check(rc: int, handle=None):
    if rc != 0:
        msg = lib().sgnb_last_error(handle)
        raise SgnbError(rc, msg.decode() if msg else "")


def fr_tables(P: int = 4, points: int = POINTS_GLL) -> dict:
    """FROperators1D(P, pointSet) tables built by the library's host set-up (no device
    needed)."""
    n = P + 1
    out = {k: np.zeros(n) for k in ("nodes", "lL", "lR", "gLp", "gRp", "qw")}
    out["D"] = np.zeros(n * n)
    _check(lib().sgnb_fr_tables_points(P, points, *(_ptr(out[k]) for k in
                                                     ("nodes", "D", "lL", "lR", "gLp", "gRp",
                                                      "qw"))))
    return out


class _DescHolder:
    """Builds an sgnb_desc and keeps the numpy arrays it points to alive."""

    def __init__(self, P, Nx, Ny, Lx, Ly, g, c, gamma, nManning, bc_x, bc_y, precision,
                 device, bathy_kind, bathy_par, tables, bathy_arrays, points=POINTS_GLL):
        self.keep = []
        d = _Desc()
        lib().sgnb_desc_init(C.byref(d))
        d.point_set = points
        d.P, d.Nx, d.Ny, d.Lx, d.Ly = P, Nx, Ny, float(Lx), float(Ly)
        d.g, d.c, d.gamma, d.nManning = float(g), float(c), float(gamma), float(nManning)
        d.bc_x, d.bc_y, d.precision, d.device = bc_x, bc_y, precision, device
        if tables is not None:
            for k in ("nodes", "D", "lL", "lR", "gLp", "gRp", "qw"):
                if k in tables:
                    a = np.ascontiguousarray(tables[k], dtype=np.float64)
                    self.keep.append(a)
                    setattr(d, k, _ptr(a))
        if bathy_arrays is not None:
            d.bathy_kind = BATHY_ARRAYS
            for k in ("Hnod", "Hx", "Hy", "HfaceX", "HfaceY", "HfaceXEnd", "HfaceYEnd"):
                if bathy_arrays.get(k) is not None:
                    a = np.ascontiguousarray(bathy_arrays[k], dtype=np.float64)
                    self.keep.append(a)
                    setattr(d, k, _ptr(a))
        else:
            d.bathy_kind = bathy_kind
            bp = np.ascontiguousarray(np.asarray(bathy_par, dtype=np.float64).reshape(-1))
            if bp.size:
                self.keep.append(bp)
                d.bathy_par = _ptr(bp)
                d.n_bathy_par = int(bp.size)
        self.desc = d


def setup_bathymetry(P=4, Nx=8, Ny=6, Lx=10.0, Ly=8.0, bathy_kind=BATHY_NONE, bathy_par=(),
                     bc_x=BC_PERIODIC, bc_y=BC_PERIODIC) -> dict:
    """The bathymetry statics the library would upload (host only, no device)."""
    h = _DescHolder(P, Nx, Ny, Lx, Ly, 9.81, 0.0, 1.5, 0.0, bc_x, bc_y, FP64_EXACT, 0,
                    bathy_kind, bathy_par, None, None)
    Nd, nf = 25 * Nx * Ny, 5 * Nx * Ny
    out = dict(Hnod=np.zeros(Nd), Hx=np.zeros(Nd), Hy=np.zeros(Nd), HfaceX=np.zeros(nf),
               HfaceY=np.zeros(nf), HfaceXEnd=np.zeros(5 * Ny), HfaceYEnd=np.zeros(5 * Nx))
    _check(lib().sgnb_setup_bathymetry(C.byref(h.desc), *(_ptr(out[k]) for k in (
        "Hnod", "Hx", "Hy", "HfaceX", "HfaceY", "HfaceXEnd", "HfaceYEnd"))))
    return out


class _DeviceArray:
    """A raw device pointer exposed through __cuda_array_interface__ (float64, 1-D)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = dict(shape=(n,), typestr="<f8", data=(ptr, False),
                                             version=3, strides=None)


class SGN2DB200:
    """Device solver with the interface of sgn::SGN2DCuda / sgn::SGN2D.

    ``precision`` FP64_EXACT reproduces the CPU reference bit for bit; FP64_FAST uses FMA
    and reciprocals (agreement within 1e-13 relative). ``tables`` / ``bathy_arrays`` take
    the arrays of a reference ``SGN2D`` (ops() and stillDepth*() accessors) so the device
    sees exactly the host's set-up, as the reference GPU solver does
    (src/cuda/sgn2d_cuda.cu:318-400); otherwise both are built by the library.
    """

    def __init__(self, P=4, Nx=8, Ny=6, Lx=10.0, Ly=8.0, g=9.81, c=0.0, gamma=1.5,
                 nManning=0.0, bc_x=BC_PERIODIC, bc_y=BC_PERIODIC, precision=FP64_EXACT,
                 device=0, bathy_kind=BATHY_NONE, bathy_par=(), tables=None,
                 bathy_arrays=None, points=POINTS_GLL, _handle=None):
        self._h = None
        self._owned = _handle is None
        if _handle is None:
            holder = _DescHolder(P, Nx, Ny, Lx, Ly, g, c, gamma, nManning, bc_x, bc_y,
                                 precision, device, bathy_kind, bathy_par, tables, bathy_arrays,
                                 points)
            h = C.c_void_p()
            _check(lib().sgnb_create(C.byref(holder.desc), C.byref(h)))
        else:
            h = C.c_void_p(_handle)
        self._h = h
        self.P, self.Nx, self.Ny, self.Lx, self.Ly = P, Nx, Ny, Lx, Ly
        self.Nd = int(lib().sgnb_ndof(h))
        self.n = 5 * self.Nd
        self.precision = precision
        self.device = device
        self.points = points

    def close(self):
        if self._h and self._owned:
            lib().sgnb_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # --- sizes and set-up (SGN2D) --------------------------------------------
    def nDof(self) -> int:
        return self.Nd

    def nTotal(self) -> int:
        return self.n

    def node_coords(self):
        x, y = np.zeros(self.Nd), np.zeros(self.Nd)
        _check(lib().sgnb_node_coords(self._h, _ptr(x), _ptr(y)), self._h)
        return x, y

    @staticmethod
    def make_state(h, u, v, w, p):
        """SGN2D::makeState (src/solver/sgn2d.cpp:107-120)."""
        h = np.asarray(h, dtype=np.float64)
        return np.concatenate([h, h * u, h * v, h * w, h * p]).astype(np.float64)

    # --- state transfer (SGN2DCuda) --------------------------------------------
    def upload(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.size != self.n:
            raise ValueError("SGN2DB200.upload: size mismatch")
        _check(lib().sgnb_upload(self._h, _ptr(U)), self._h)

    def download(self, out=None):
        if out is None:
            out = np.empty(self.n)
        elif not (isinstance(out, np.ndarray) and out.size == self.n and out.flags["WRITEABLE"]):
            raise ValueError("SGN2DB200.download: out must be a writable array of 5 * nDof doubles")
        _check(lib().sgnb_download(self._h, _ptr(out)), self._h)
        return out

    # --- right-hand side -------------------------------------------------------
    def rhs_once(self):
        """R(uploaded state), downloaded (SGN2DCuda::rhsOnce)."""
        dU = np.empty(self.n)
        _check(lib().sgnb_rhs_once(self._h, _ptr(dU)), self._h)
        return dU

    def rhs(self, U):
        """R(U) for a host array, stateless (SGN2D::rhs)."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.size != self.n:
            raise ValueError("SGN2D::rhs: size mismatch")
        dU = np.empty(self.n)
        _check(lib().sgnb_rhs_host(self._h, _ptr(U), _ptr(dU)), self._h)
        return dU

    def rhs_device(self, U_ptr: int, dU_ptr: int, stream: int | None = None):
        """R(U) for device pointers (e.g. torch tensors' data_ptr()), asynchronous.

        stream None runs on the context stream; an integer is a cudaStream_t, and 0 (the
        handle torch reports for its default stream) means the legacy default stream."""
        if stream is None:
            s = None
        else:
            s = C.c_void_p(stream if stream else _CUDA_STREAM_LEGACY)
        _check(lib().sgnb_rhs_device(self._h, C.c_void_p(U_ptr), C.c_void_p(dU_ptr), s),
               self._h)

    def state_device_ptr(self):
        u, s = C.c_void_p(), C.c_void_p()
        _check(lib().sgnb_state_device_ptr(self._h, C.byref(u), C.byref(s)), self._h)
        return u.value, s.value

    def state_tensor(self):
        """The current device state as a float64 torch tensor view (no copy). Valid until
        the next integration (which may switch the state buffer); the library works on its
        own stream, so synchronise before reading or writing it from torch."""
        import torch

        u, _ = self.state_device_ptr()
        return torch.as_tensor(_DeviceArray(u, self.n), device=f"cuda:{self.device}")

    def upload_tensor(self, t):
        """Device-to-device upload of a float64 torch tensor holding a state."""
        import torch

        if t.dtype != torch.float64 or t.numel() != self.n:
            raise ValueError("SGN2DB200.upload_tensor: float64 tensor of size 5 * nDof expected")
        torch.cuda.synchronize(self.device)
        self.state_tensor().copy_(t.reshape(-1))
        torch.cuda.synchronize(self.device)

    # --- integrators -------------------------------------------------------------
    def integrate_adaptive(self, t0, tEnd, dt0, opt: AdaptiveRKOptions | None = None,
                           raise_on_nan=True) -> AdaptiveRKStats:
        """SGN2DCuda::integrateAdaptive: device-resident BS3(2) of the uploaded state."""
        o = _Opts(**dataclasses.asdict(opt or AdaptiveRKOptions()))
        st = _Stats()
        rc = lib().sgnb_integrate_adaptive(self._h, t0, tEnd, dt0, C.byref(o), C.byref(st))
        if rc != 0 and (raise_on_nan or rc != 4):
            _check(rc, self._h)
        return AdaptiveRKStats(st.accepted, st.rejected, st.rhsEvals, st.attempts,
                               st.tReached, st.dtLast, st.maxNormLast, st.aborted,
                               st.kernel_launches)

    def integrate_steps(self, t0, dt0, nsteps, opt: AdaptiveRKOptions | None = None
                        ) -> AdaptiveRKStats:
        """The device-resident loop for a fixed number of accepted steps."""
        o = _Opts(**dataclasses.asdict(opt or AdaptiveRKOptions()))
        st = _Stats()
        _check(lib().sgnb_integrate_steps(self._h, t0, dt0, int(nsteps), C.byref(o),
                                          C.byref(st)), self._h)
        return AdaptiveRKStats(st.accepted, st.rejected, st.rhsEvals, st.attempts,
                               st.tReached, st.dtLast, st.maxNormLast, st.aborted,
                               st.kernel_launches)

    def launch_stage(self, stage: int, dt: float, count: int = 1, stream: int | None = None):
        """Profiling hook: `count` launches of one fused stage kernel (2, 3 or 4)."""
        s = None if stream is None else C.c_void_p(stream if stream else _CUDA_STREAM_LEGACY)
        _check(lib().sgnb_launch_stage(self._h, stage, dt, count, s), self._h)

    def bs3_steps(self, t0, dts):
        """Consecutive bs3Step calls with the given step sizes (frozen-dt replay)."""
        d = np.ascontiguousarray(dts, dtype=np.float64)
        _check(lib().sgnb_bs3_steps(self._h, t0, _ptr(d), int(d.size)), self._h)

    def rk4_steps(self, t0, dts):
        """Consecutive rk4Step calls (classical RK4, rk.cpp:23-38) with the given step
        sizes; FP64 modes."""
        d = np.ascontiguousarray(dts, dtype=np.float64)
        _check(lib().sgnb_rk4_steps(self._h, t0, _ptr(d), int(d.size)), self._h)

    def attempt_log(self, cap=1 << 16):
        """Rows (t, dt, errNorm, accepted) of the last integration's attempts."""
        buf = np.zeros(4 * cap)
        n = C.c_longlong()
        _check(lib().sgnb_attempt_log(self._h, _ptr(buf), cap, C.byref(n)), self._h)
        return buf[: 4 * min(n.value, cap)].reshape(-1, 4)

    def rhs_vjp(self, U, Rbar):
        """(dR/dU)^T Rbar at the host state U and the cotangents of the depth statics
        (dict with the keys of setup_bathymetry)."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        Rbar = np.ascontiguousarray(Rbar, dtype=np.float64)
        if U.size != self.n or Rbar.size != self.n:
            raise ValueError("rhs_vjp: U and Rbar must hold 5 * nDof values")
        Ub = np.empty(self.n)
        Nd, nf = self.Nd, 5 * self.Nx * self.Ny
        bars = dict(Hnod=np.zeros(Nd), Hx=np.zeros(Nd), Hy=np.zeros(Nd), HfaceX=np.zeros(nf),
                    HfaceY=np.zeros(nf), HfaceXEnd=np.zeros(5 * self.Ny),
                    HfaceYEnd=np.zeros(5 * self.Nx))
        _check(lib().sgnb_rhs_vjp(self._h, _ptr(U), _ptr(Rbar), _ptr(Ub), *(_ptr(bars[k]) for k in (
            "Hnod", "Hx", "Hy", "HfaceX", "HfaceY", "HfaceXEnd", "HfaceYEnd"))), self._h)
        return Ub, bars

    # --- diagnostics -------------------------------------------------------------
    def _scalar(self, fn, *args):
        out = C.c_double()
        _check(fn(self._h, *args, C.byref(out)), self._h)
        return out.value

    def max_wave_speed(self):
        return self._scalar(lib().sgnb_max_wave_speed)

    def cfl_time_step(self, cfl):
        return self._scalar(lib().sgnb_cfl_time_step, C.c_double(cfl))

    def mass(self):
        return self._scalar(lib().sgnb_mass)

    def energy(self):
        return self._scalar(lib().sgnb_energy)

    def eta_max(self, window=None):
        """Largest eta = h - H of the current state inside window (x0, x1, y0, y1), the
        whole domain by default, and its node index (-1 when the window holds no node)."""
        inf = float("inf")
        x0, x1, y0, y1 = window if window is not None else (-inf, inf, -inf, inf)
        v = C.c_double()
        n = C.c_longlong()
        _check(lib().sgnb_eta_max(self._h, x0, x1, y0, y1, C.byref(v), C.byref(n)), self._h)
        return v.value, n.value

    def sample_eta(self, nodes):
        """eta at the given node indices (gauges)."""
        nd = np.ascontiguousarray(nodes, dtype=np.int64)
        out = np.zeros(nd.size)
        _check(lib().sgnb_sample_eta(self._h, nd.ctypes.data_as(C.POINTER(C.c_longlong)),
                                     int(nd.size), _ptr(out)), self._h)
        return out

    def element_means(self):
        """Element means of (eta, u, v, p, H), shape [5, Ny, Nx]."""
        out = np.zeros(5 * self.Nx * self.Ny)
        _check(lib().sgnb_element_means(self._h, _ptr(out)), self._h)
        return out.reshape(5, self.Ny, self.Nx)

    def write_vtk(self, path):
        """Legacy-VTK frame of the element means (the reference's vtk2d.h format)."""
        _check(lib().sgnb_write_vtk(self._h, os.fsencode(path)), self._h)

    def nearest_node(self, x, y):
        n = C.c_longlong()
        _check(lib().sgnb_nearest_node(self._h, float(x), float(y), C.byref(n)), self._h)
        return n.value


def _stats(st) -> AdaptiveRKStats:
    return AdaptiveRKStats(st.accepted, st.rejected, st.rhsEvals, st.attempts, st.tReached,
                           st.dtLast, st.maxNormLast, st.aborted, st.kernel_launches)


class SGNBatch:
    """Many independent SGN2D instances advanced together (FP64_FAST, or MIXED with
    ``precision=MIXED``).

    ``instances`` is a list of keyword dicts for SGN2DB200 (mesh size, domain, c, gamma,
    boundaries, bathymetry). Every RK stage is one persistent launch over the tiles of all
    instances; each instance keeps its own adaptive controller. ``self[i]`` is a view of
    instance i with the single-instance methods (upload, download, rhs, mass, ...).
    """

    def __init__(self, instances, device=0, precision=FP64_FAST):
        self._b = None
        holders = []
        for kw in instances:
            kw = dict(kw)
            kw.setdefault("precision", precision)
            kw["device"] = device
            args = [kw.pop(k, dflt) for k, dflt in (
                ("P", 4), ("Nx", 8), ("Ny", 6), ("Lx", 10.0), ("Ly", 8.0), ("g", 9.81),
                ("c", 0.0), ("gamma", 1.5), ("nManning", 0.0), ("bc_x", BC_PERIODIC),
                ("bc_y", BC_PERIODIC), ("precision", FP64_FAST), ("device", 0),
                ("bathy_kind", BATHY_NONE), ("bathy_par", ()), ("tables", None),
                ("bathy_arrays", None), ("points", POINTS_GLL))]
            if kw:
                raise TypeError(f"SGNBatch: unknown instance keys {sorted(kw)}")
            holders.append(_DescHolder(*args))
        n = len(holders)
        descs = (_Desc * n)(*[h.desc for h in holders])
        b = C.c_void_p()
        rc = lib().sgnb_batch_create(descs, n, C.byref(b))
        if rc != 0:
            msg = lib().sgnb_batch_last_error(None)
            raise SgnbError(rc, msg.decode() if msg else "")
        self._b = b
        self.n = n
        self._views = []
        for i, h in enumerate(holders):
            d = h.desc
            self._views.append(SGN2DB200(P=d.P, Nx=d.Nx, Ny=d.Ny, Lx=d.Lx, Ly=d.Ly,
                                         precision=d.precision, device=device,
                                         _handle=lib().sgnb_batch_instance(b, i)))

    def _check(self, rc):
        if rc != 0:
            msg = lib().sgnb_batch_last_error(self._b)
            raise SgnbError(rc, msg.decode() if msg else "")

    def close(self):
        if self._b:
            for v in self._views:
                v.close()
            lib().sgnb_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __len__(self):
        return self.n

    def __getitem__(self, i) -> SGN2DB200:
        return self._views[i]

    def integrate_steps(self, dt0, nsteps, opt: AdaptiveRKOptions | None = None):
        """``nsteps`` accepted BS3(2) steps of every instance from step sizes ``dt0[i]``."""
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dt0, dtype=np.float64), (self.n,)))
        o = _Opts(**dataclasses.asdict(opt or AdaptiveRKOptions()))
        st = (_Stats * self.n)()
        self._check(lib().sgnb_batch_integrate_steps(self._b, _ptr(d), int(nsteps), C.byref(o),
                                                     st))
        return [_stats(s) for s in st]

    @property
    def stream(self) -> int:
        """The batch's CUDA stream handle (its launches run there)."""
        sp = C.c_void_p()
        self._check(lib().sgnb_batch_stream(self._b, C.byref(sp)))
        return sp.value or 0

    @property
    def config(self):
        sh, bl = C.c_int(), C.c_int()
        self._check(lib().sgnb_batch_get_config(self._b, C.byref(sh), C.byref(bl)))
        return sh.value, bl.value

    @config.setter
    def config(self, value):
        self._check(lib().sgnb_batch_set_config(self._b, int(value[0]), int(value[1])))

    def autotune(self, dt0, reps=3):
        """Times every (tile shape, grid) pair; keeps the fastest. Returns ms per attempt,
        [3 shapes (8x4, 16x2, 4x8), 5 grids (one CTA per tile, 1..4 persistent CTAs per
        SM)]."""
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dt0, dtype=np.float64), (self.n,)))
        ms = np.zeros(15)
        self._check(lib().sgnb_batch_autotune(self._b, _ptr(d), int(reps), _ptr(ms)))
        return ms.reshape(3, 5)
