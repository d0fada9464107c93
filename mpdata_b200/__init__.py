"""mpdata_b200 -- MPDATA transport step on NVIDIA B200, Python bindings.

Thin ctypes layer over ``libmpdata_b200.so`` (the C ABI declared in
``include/mpdata_b200.h``).  There is no CPU fallback: importing this module
fails if the compiled library is missing, and every call runs the CUDA
kernels.

Two levels, mirroring the C ABI:

* :func:`smolar` / :func:`msmolar` / :func:`msmolar_gather` -- the reference
  library's entry points (apc-llc/mpdata ``smolar.h:45-48,95-99,132-136``)
  on numpy host arrays, with the reference's pointer exchange expressed as the
  returned ``(c0, c1)`` pair;
* :class:`Solver` -- the device-resident handle API (``mpdata_*``).

Arrays are full grids of shape ``(ns, ny, nx)``, x fastest, shell included.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmpdata_b200.so")

SOLENOIDAL, DIVERGENT = 0, 1
MSMOLAR_SERIAL, MSMOLAR_PTHREADS, MSMOLAR_OPENMP = 0, 1, 2
F32, F64 = 0, 1
HOST, DEVICE, HOST_ASYNC, DEVICE_BORROW = 0, 1, 2, 3
DIV_REFERENCE, DIV_OFF = 0, 1

ERRORS = {-1: "MPDATA_ERR_ARG", -2: "MPDATA_ERR_CUDA", -3: "MPDATA_ERR_NOMEM",
          -4: "MPDATA_ERR_COURANT", -5: "MPDATA_ERR_STATE", -6: "MPDATA_ERR_INT_DIV0"}


class MpdataError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `make -C mpdata_b200/csrc` "
        "(or __graft_entry__.build()); there is no CPU fallback")

_lib = C.CDLL(LIB_PATH)


class Options(C.Structure):
    """struct mpdata_options (include/mpdata_b200.h)."""
    _fields_ = [("limiter", C.c_int), ("precision_form", C.c_int), ("div_mode", C.c_int),
                ("vv_fix", C.c_int), ("strict", C.c_int), ("kernel", C.c_int),
                ("check_courant", C.c_int), ("approx_div", C.c_int)]


_vp = C.c_void_p
_lib.mpdata_last_error.restype = C.c_char_p
_lib.mpdata_create.argtypes = [C.POINTER(_vp), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                               C.POINTER(Options)]
_lib.mpdata_destroy.argtypes = [_vp]
_lib.mpdata_set_stream.argtypes = [_vp, _vp]
_lib.mpdata_set_velocity.argtypes = [_vp, _vp, _vp, _vp, C.c_double] + [_vp] * 6 + [C.c_int]
_lib.mpdata_set_faces.argtypes = [_vp, _vp, _vp, _vp, C.c_int]
_lib.mpdata_set_field.argtypes = [_vp, _vp, C.c_int]
_lib.mpdata_get_field.argtypes = [_vp, _vp, C.c_int]
_lib.mpdata_get_previous.argtypes = [_vp, _vp, C.c_int]
_lib.mpdata_step.argtypes = [_vp, C.c_int]
_lib.mpdata_get_planes.argtypes = [_vp, C.c_int, C.c_int, _vp, C.c_int]
_lib.mpdata_set_planes.argtypes = [_vp, C.c_int, C.c_int, _vp, C.c_int]
_lib.mpdata_sync.argtypes = [_vp]
_lib.mpdata_wait.argtypes = [_vp, C.c_int]
_lib.mpdata_mass.argtypes = [_vp, C.POINTER(C.c_double)]
_lib.mpdata_min.argtypes = [_vp, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]
_lib.mpdata_launches_per_step.argtypes = [_vp]
_lib.mpdata_host_alloc.restype = _vp
_lib.mpdata_host_alloc.argtypes = [C.c_size_t]
_lib.mpdata_host_free.argtypes = [_vp]
_lib.msmolar_free.argtypes = [C.POINTER(_vp)]
_lib.mpdata_set_default_options.argtypes = [C.POINTER(Options)]
_lib.mpdata_set_pipeline.argtypes = [C.c_int]
_lib.mpdata_ensemble_create.argtypes = [C.POINTER(_vp), C.c_int, C.POINTER(C.c_int),
                                        C.POINTER(C.c_int), C.c_int, C.POINTER(Options)]
_lib.mpdata_ensemble_destroy.argtypes = [_vp]
_lib.mpdata_ensemble_set_stream.argtypes = [_vp, _vp]
_lib.mpdata_ensemble_set_faces.argtypes = [_vp, C.c_int, _vp, _vp, C.c_int]
_lib.mpdata_ensemble_set_field.argtypes = [_vp, C.c_int, _vp, C.c_int]
_lib.mpdata_ensemble_get_field.argtypes = [_vp, C.c_int, _vp, C.c_int]
_lib.mpdata_ensemble_step.argtypes = [_vp, C.c_int]
_lib.mpdata_ensemble_step_direct.argtypes = [_vp, C.c_int]
_lib.mpdata_ensemble_sync.argtypes = [_vp]
_lib.mpdata_ensemble_autotune.argtypes = [_vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]
_lib.mpdata_ensemble_tile.argtypes = [_vp, C.c_int]
_lib.mpdata_set_march_depth.argtypes = [_vp, C.c_int]
_lib.mpdata_march_depth.argtypes = [_vp]
_lib.mpdata_autotune.argtypes = [_vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]
_lib.mpdata_enable_pass_timing.argtypes = [_vp, C.c_int]
_lib.mpdata_pass_times.argtypes = [_vp, C.POINTER(C.c_double * 3), C.POINTER(C.c_longlong * 3),
                                   C.c_int]


_lib.mpdata_check_division.argtypes = [C.c_longlong, C.c_ulonglong, C.POINTER(C.c_longlong)]


def check_division(n: int, seed: int = 1) -> int:
    """Bitwise mismatches between the two-cell pass's division and IEEE
    division on n seeded random operand pairs (``mpdata_check_division``)."""
    out = C.c_longlong(-1)
    _check(_lib.mpdata_check_division(n, seed, C.byref(out)))
    return out.value


def last_error() -> str:
    return _lib.mpdata_last_error().decode()


def _check(rc: int) -> int:
    if rc < 0:
        raise MpdataError(rc, last_error())
    return rc


def library() -> C.CDLL:
    """The loaded C library (for direct C-ABI calls)."""
    return _lib


def set_default_options(options: "SolverOptions | None" = None) -> None:
    """Options for :func:`smolar`/:func:`msmolar` on the calling thread
    (``mpdata_set_default_options``); None restores the reference defaults."""
    if options is None:
        _check(_lib.mpdata_set_default_options(None))
    else:
        o = options.to_c()
        _check(_lib.mpdata_set_default_options(C.byref(o)))


def set_pipeline(chunk_planes: int = 0) -> None:
    """z planes per chunk of the pipelined :func:`smolar` host step on the
    calling thread (``mpdata_set_pipeline``): 0 automatic, < 0 no pipelining."""
    _check(_lib.mpdata_set_pipeline(int(chunk_planes)))


def _dtype_code(dtype) -> int:
    dt = np.dtype(dtype)
    if dt == np.float32:
        return F32
    if dt == np.float64:
        return F64
    raise TypeError(f"unsupported dtype {dt}")


def _ctype(dtype):
    dt = np.dtype(dtype)
    if dt == np.int64:
        return C.c_long  # the reference's INTEGER build: real = long
    return C.c_float if dt == np.float32 else C.c_double


def _host_ptr(a: np.ndarray, dtype) -> C.c_void_p:
    if not isinstance(a, np.ndarray):
        raise TypeError("host array expected")
    if a.dtype != np.dtype(dtype) or not a.flags.c_contiguous:
        raise TypeError(f"expected a C-contiguous {np.dtype(dtype)} array, got {a.dtype}")
    return C.c_void_p(a.ctypes.data)


def _ptr(a, dtype):
    """(pointer, where) of a numpy host array or a CUDA tensor (torch)."""
    if isinstance(a, np.ndarray):
        return _host_ptr(a, dtype), HOST
    if hasattr(a, "data_ptr") and getattr(a, "is_cuda", False):
        if not a.is_contiguous():
            raise TypeError("device tensor must be contiguous")
        return C.c_void_p(a.data_ptr()), DEVICE
    if hasattr(a, "data_ptr"):  # CPU tensor
        return C.c_void_p(a.data_ptr()), HOST
    raise TypeError(f"unsupported array type {type(a)}")


# ---------------------------------------------------------------------------
# reference entry points

def smolar(nx, ny, ns, dx, dy, ds, dt, u0, u1, v0, v1, w0, w1, c0, c1,
           flow_type=DIVERGENT, order=2, dtype=np.float32):
    """One MPDATA step through the reference-compatible ``smolar()``
    (``smolar_f64()`` for float64, ``smolar_i64()`` -- the reference's
    INTEGER build -- for int64, where ``dt`` is an integer too).

    ``c0`` is the input field and both ``c0`` and ``c1`` are written.  Returns
    ``(c0, c1)`` the way the reference leaves ``*c0``/``*c1``: ``c1`` is the
    newest field, ``c0`` the field before the last pass (the two arrays trade
    places iff ``order`` is even, core/src/smolar.c:58)."""
    fn = {np.dtype(np.float32): _lib.smolar, np.dtype(np.float64): _lib.smolar_f64,
          np.dtype(np.int64): _lib.smolar_i64}[np.dtype(dtype)]
    T = _ctype(dtype)
    if np.dtype(dtype) == np.int64:
        dt = int(dt)
    P = C.POINTER(T)
    pc0 = C.cast(c0.ctypes.data, P)
    pc1 = C.cast(c1.ctypes.data, P)
    args = [_host_ptr(x, dtype) for x in (dx, dy, ds)]
    vel = [_host_ptr(x, dtype) for x in (u0, u1, v0, v1, w0, w1)]
    rc = fn(C.c_int(nx), C.c_int(ny), C.c_int(ns), *args, T(dt), *vel, C.byref(pc0),
            C.byref(pc1), C.c_int(flow_type), C.c_int(order))
    _check(rc)
    by_addr = {c0.ctypes.data: c0, c1.ctypes.data: c1}
    return (by_addr[C.cast(pc0, C.c_void_p).value], by_addr[C.cast(pc1, C.c_void_p).value])


class MsmolarState:
    """Holds the ``void* desc`` of the decomposed solver (reference smolar.h:95-99)."""

    def __init__(self):
        self.desc = C.c_void_p(None)

    def free(self):
        if self.desc.value:
            _check(_lib.msmolar_free(C.byref(self.desc)))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _msmolar_call(fn, state, nx, ny, ns, dx, dy, ds, dt, u0, u1, v0, v1, w0, w1, c0, c1,
                  flow_type, order, sx, sy, ss, mode):
    P = C.POINTER(C.c_float)
    pc0 = C.cast(c0.ctypes.data, P)
    pc1 = C.cast(c1.ctypes.data, P)
    args = [_host_ptr(x, np.float32) for x in (dx, dy, ds)]
    vel = [_host_ptr(x, np.float32) for x in (u0, u1, v0, v1, w0, w1)]
    rc = fn(C.byref(state.desc), C.c_int(nx), C.c_int(ny), C.c_int(ns), *args, C.c_float(dt),
            *vel, C.byref(pc0), C.byref(pc1), C.c_int(flow_type), C.c_int(order), C.c_int(sx),
            C.c_int(sy), C.c_int(ss), C.c_int(mode))
    _check(rc)
    by_addr = {c0.ctypes.data: c0, c1.ctypes.data: c1}
    return (by_addr[C.cast(pc0, C.c_void_p).value], by_addr[C.cast(pc1, C.c_void_p).value])


def msmolar(state: MsmolarState, nx, ny, ns, dx, dy, ds, dt, u0, u1, v0, v1, w0, w1, c0, c1,
            flow_type=DIVERGENT, order=2, sx=1, sy=1, ss=1, mode=MSMOLAR_SERIAL):
    """Decomposed step (float32).  Returns the exchanged ``(c0, c1)`` pair; the
    arrays' contents are refreshed only by :func:`msmolar_gather`."""
    return _msmolar_call(_lib.msmolar, state, nx, ny, ns, dx, dy, ds, dt, u0, u1, v0, v1, w0,
                         w1, c0, c1, flow_type, order, sx, sy, ss, mode)


def msmolar_gather(state: MsmolarState, nx, ny, ns, dx, dy, ds, dt, u0, u1, v0, v1, w0, w1,
                   c0, c1, flow_type=DIVERGENT, order=2, sx=1, sy=1, ss=1,
                   mode=MSMOLAR_SERIAL):
    """Copy the decomposed state's newest field into ``c1`` (previous into ``c0``)."""
    return _msmolar_call(_lib.msmolar_gather, state, nx, ny, ns, dx, dy, ds, dt, u0, u1, v0,
                         v1, w0, w1, c0, c1, flow_type, order, sx, sy, ss, mode)


# ---------------------------------------------------------------------------
# handle API

@dataclass
class SolverOptions:
    limiter: bool = False
    precision_form: bool = False
    div_mode: int = DIV_REFERENCE
    vv_fix: bool = False
    strict: bool = False
    # 0 fused per-pass kernels (the faster form for the options), 1 one kernel per
    # reference routine, 2 fused with one cell per thread, 3 fused with two cells
    # per thread (float32 without strict / precision_form)
    kernel: int = 0
    check_courant: bool = False
    approx_div: bool = False

    def to_c(self) -> Options:
        return Options(int(self.limiter), int(self.precision_form), int(self.div_mode),
                       int(self.vv_fix), int(self.strict), int(self.kernel),
                       int(self.check_courant), int(self.approx_div))


class Solver:
    """Device-resident MPDATA solver (``mpdata_create`` ... ``mpdata_destroy``)."""

    def __init__(self, nx: int, ny: int, ns: int, order: int = 2, dtype=np.float32,
                 options: SolverOptions | None = None, **kw):
        opts = options or SolverOptions(**kw)
        self.nx, self.ny, self.ns, self.order = nx, ny, ns, order
        self.dtype = np.dtype(dtype)
        self.options = opts
        self._h = C.c_void_p(None)
        o = opts.to_c()
        _check(_lib.mpdata_create(C.byref(self._h), nx, ny, ns, _dtype_code(dtype), order,
                                  C.byref(o)))

    @property
    def shape(self):
        return (self.ns, self.ny, self.nx)

    def close(self):
        if self._h and self._h.value:
            _lib.mpdata_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_stream(self, stream_handle: int | None):
        _check(_lib.mpdata_set_stream(self._h, C.c_void_p(stream_handle)))

    def set_velocity(self, dx, dy, ds, dt, u0, u1, v0, v1, w0, w1, borrow: bool = False):
        """``borrow``: CUDA tensors the handle reads in place until the next
        step has run (MPDATA_DEVICE_BORROW); leave them unchanged until then."""
        ptrs = [_ptr(x, self.dtype) for x in (dx, dy, ds, u0, u1, v0, v1, w0, w1)]
        wheres = {w for _, w in ptrs}
        if len(wheres) != 1:
            raise TypeError("all velocity arguments must live in the same memory")
        where = wheres.pop()
        if borrow:
            if where != DEVICE:
                raise TypeError("only device arrays can be lent")
            where = DEVICE_BORROW
        p = [x for x, _ in ptrs]
        _check(_lib.mpdata_set_velocity(self._h, p[0], p[1], p[2], C.c_double(dt), *p[3:], where))

    def set_faces(self, U, V, W):
        ptrs = [_ptr(x, self.dtype) for x in (U, V, W)]
        _check(_lib.mpdata_set_faces(self._h, ptrs[0][0], ptrs[1][0], ptrs[2][0], ptrs[0][1]))

    def set_field(self, c):
        p, where = _ptr(c, self.dtype)
        _check(_lib.mpdata_set_field(self._h, p, where))

    def get_field(self, out=None, previous: bool = False):
        if out is None:
            out = np.empty(self.shape, self.dtype)
        p, where = _ptr(out, self.dtype)
        fn = _lib.mpdata_get_previous if previous else _lib.mpdata_get_field
        _check(fn(self._h, p, where))
        return out

    def step(self, nsteps: int = 1):
        _check(_lib.mpdata_step(self._h, nsteps))

    def get_planes(self, k0: int, nk: int, out=None):
        """z-planes [k0, k0+nk) of the newest field (``mpdata_get_planes``);
        ``out``: a host array or a CUDA tensor of shape (nk, ny, nx)."""
        if out is None:
            out = np.empty((nk,) + self.shape[1:], self.dtype)
        p, where = _ptr(out, self.dtype)
        _check(_lib.mpdata_get_planes(self._h, k0, nk, p, where))
        return out

    def get_planes_async(self, k0: int, nk: int, out) -> int:
        """Queue the copy of z-planes [k0, k0+nk) into ``out``, a C-contiguous
        (nk, ny, nx) view of pinned host memory (``mpdata_host_alloc``), and
        return its ticket: ``out`` holds the planes after ``wait(ticket)``
        (``mpdata_get_planes`` with MPDATA_HOST_ASYNC)."""
        if not (isinstance(out, np.ndarray) and out.dtype == self.dtype and out.flags.c_contiguous
                and out.shape == (nk,) + self.shape[1:]):
            raise TypeError("expected a C-contiguous host array of shape (nk, ny, nx)")
        return _check(_lib.mpdata_get_planes(self._h, k0, nk, C.c_void_p(out.ctypes.data),
                                             HOST_ASYNC))

    def wait(self, ticket: int):
        """Wait for a queued copy (``mpdata_wait``)."""
        _check(_lib.mpdata_wait(self._h, ticket))

    def set_planes(self, k0: int, planes):
        """Overwrite z-planes [k0, k0+len) in every level (``mpdata_set_planes``)."""
        p, where = _ptr(planes, self.dtype)
        _check(_lib.mpdata_set_planes(self._h, k0, int(planes.shape[0]), p, where))

    def sync(self):
        _check(_lib.mpdata_sync(self._h))

    def mass(self) -> float:
        m = C.c_double()
        _check(_lib.mpdata_mass(self._h, C.byref(m)))
        return m.value

    def min(self):
        m = C.c_double()
        n = C.c_longlong()
        _check(_lib.mpdata_min(self._h, C.byref(m), C.byref(n)))
        return m.value, n.value

    def launches_per_step(self) -> int:
        return _check(_lib.mpdata_launches_per_step(self._h))

    def set_march_depth(self, depth: int):
        _check(_lib.mpdata_set_march_depth(self._h, depth))

    def march_depth(self) -> int:
        return _check(_lib.mpdata_march_depth(self._h))

    def autotune(self, trial_steps: int = 5):
        """Time the z-march depth candidates on this solver's field, keep the
        fastest; returns (depth, ms per step).  The field is restored."""
        dep = C.c_int()
        ms = C.c_double()
        _check(_lib.mpdata_autotune(self._h, trial_steps, C.byref(dep), C.byref(ms)))
        return dep.value, ms.value

    def enable_pass_timing(self, on: bool = True):
        _check(_lib.mpdata_enable_pass_timing(self._h, int(on)))

    def pass_times(self, reset: bool = False):
        """(ms, launches) per pass class: donor, corrective writing faces,
        last corrective pass (CUDA events on the handle's stream)."""
        ms = (C.c_double * 3)()
        n = (C.c_longlong * 3)()
        _check(_lib.mpdata_pass_times(self._h, C.byref(ms), C.byref(n), int(reset)))
        return list(ms), list(n)


class Ensemble:
    """Batched ensemble of independent 2D problems (``mpdata_ensemble_*``).

    Instance q is an ``ny[q] x nx[q]`` grid (the reference's 2D form:
    ``nx x ny x 3`` with w = 0), float32.  Faces and fields are 2D arrays of
    shape ``(ny, nx)``."""

    # Candidates of the autotuner: tile shapes (threads x, y) of the tile
    # kernels, and 3 = the y-march (the first corrective pass by one warp per
    # strip of 32 columns x 64 rows, the other passes with tile 1).
    TILES = ((32, 8), (32, 16), (64, 8), (32, 64))
    MARCH = 3

    def __init__(self, nx, ny, order: int = 2, options: SolverOptions | None = None, **kw):
        opts = options or SolverOptions(**kw)
        self.nx = [int(v) for v in nx]
        self.ny = [int(v) for v in ny]
        if len(self.nx) != len(self.ny):
            raise ValueError("nx and ny differ in length")
        self.n = len(self.nx)
        self.order = order
        self._h = C.c_void_p(None)
        o = opts.to_c()
        ax = (C.c_int * self.n)(*self.nx)
        ay = (C.c_int * self.n)(*self.ny)
        _check(_lib.mpdata_ensemble_create(C.byref(self._h), self.n, ax, ay, order, C.byref(o)))

    def close(self):
        if self._h and self._h.value:
            _lib.mpdata_ensemble_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_stream(self, stream_handle):
        _check(_lib.mpdata_ensemble_set_stream(self._h, C.c_void_p(stream_handle)))

    def set_faces(self, q, U, V):
        (pu, w), (pv, _) = _ptr(U, np.float32), _ptr(V, np.float32)
        _check(_lib.mpdata_ensemble_set_faces(self._h, q, pu, pv, w))

    def set_field(self, q, c):
        p, w = _ptr(c, np.float32)
        _check(_lib.mpdata_ensemble_set_field(self._h, q, p, w))

    def get_field(self, q, out=None):
        if out is None:
            out = np.empty((self.ny[q], self.nx[q]), np.float32)
        p, w = _ptr(out, np.float32)
        _check(_lib.mpdata_ensemble_get_field(self._h, q, p, w))
        return out

    def step(self, nsteps: int = 1, graph: bool = True):
        fn = _lib.mpdata_ensemble_step if graph else _lib.mpdata_ensemble_step_direct
        _check(fn(self._h, nsteps))

    def sync(self):
        _check(_lib.mpdata_ensemble_sync(self._h))

    def autotune(self, trial_steps: int = 5):
        t = C.c_int()
        ms = C.c_double()
        _check(_lib.mpdata_ensemble_autotune(self._h, trial_steps, C.byref(t), C.byref(ms)))
        return t.value, ms.value

    def set_tile(self, tile: int):
        _check(_lib.mpdata_ensemble_tile(self._h, tile))
