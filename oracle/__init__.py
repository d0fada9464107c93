"""CPU oracle for the MPDATA step -- TEST INFRASTRUCTURE ONLY.

Python (ctypes + numpy) access to

* ``liboracle.so``  -- this project's C restatement of the reference's
  ``smolar()`` path (``mpdata_oracle.c``), always buildable with gcc;
* ``_ref/libref_*.so`` -- the reference's own C sources compiled unmodified
  by ``oracle/Makefile`` (present only where the reference checkout was
  available when the build ran; the built files travel with the tree).

Only the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may use this package, and only as the checker / the timed CPU baseline.
The shipped library never imports it.

Arrays are numpy, full grids of shape ``(ns, ny, nx)`` (x fastest), exactly
the reference's memory layout (``core/src/smolar_pass.c:86``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
# The reference checkout to compile from (build time only; the built files
# travel with the tree and nothing reads the checkout at run time).
REFERENCE_SRC = os.environ.get("MPDATA_REFERENCE_SRC")


class OracleOpts(C.Structure):
    _fields_ = [("limiter", C.c_int), ("vv_fix", C.c_int), ("div_mode", C.c_int),
                ("wide_beta", C.c_int)]


def build(reference: bool = True, reference_src: str | None = None) -> None:
    """Compile liboracle.so, and the reference libraries when a reference
    checkout is given (`reference_src`, else $MPDATA_REFERENCE_SRC) and
    present; without one the reference build is skipped."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    src = reference_src or REFERENCE_SRC
    if reference and src and os.path.isdir(os.path.join(src, "core", "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={src}"], check=True)
        # the reference's ring drivers, also linked against the GPU library once it is built
        lib = os.path.join(os.path.dirname(HERE), "mpdata_b200", "libmpdata_b200.so")
        if os.path.exists(lib):
            subprocess.run(["make", "-s", "-C", HERE, "drivers", f"REF={src}"],
                           check=True)


_libs: dict[str, C.CDLL] = {}


def _load(path: str) -> C.CDLL:
    if path not in _libs:
        _libs[path] = C.CDLL(path)
    return _libs[path]


def oracle_lib() -> C.CDLL:
    path = os.path.join(HERE, "liboracle.so")
    if not os.path.exists(path):
        build(reference=False)
    return _load(path)


def ref_available(variant: str = "f32") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_{variant}.so"))


def ref_lib(variant: str = "f32") -> C.CDLL:
    """variant: 'f32' / 'f64' (strict IEEE) or 'f32_fast' (reference CMake flags)."""
    path = os.path.join(REF_DIR, f"libref_{variant}.so")
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    return _load(path)


def _ct(dtype):
    """C type of `real`: float, double, or long (the INTEGER build)."""
    dt = np.dtype(dtype)
    if dt == np.int64:
        return C.c_long
    return C.c_float if dt == np.float32 else C.c_double


def _p(a: np.ndarray, dtype):
    assert a.dtype == np.dtype(dtype) and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(_ct(dtype)))


def _sfx(dtype) -> str:
    dt = np.dtype(dtype)
    if dt == np.int64:
        return "i64"
    return "f32" if dt == np.float32 else "f64"


def opts(limiter=0, vv_fix=0, div_mode=0, wide_beta=0) -> OracleOpts:
    return OracleOpts(limiter, vv_fix, div_mode, wide_beta)


def _smolar_call(fn, dtype, dx, dy, ds, dt, u0, u1, v0, v1, w0, w1, c0, c1, order,
                 extra=()):
    """Run a smolar()-signature function; returns (rc, newest, other) following
    the returned pointer order (smolar.c:58)."""
    ns, ny, nx = c0.shape
    T = _ct(dtype)
    pc0 = C.cast(c0.ctypes.data, C.POINTER(T))
    pc1 = C.cast(c1.ctypes.data, C.POINTER(T))
    dt = int(dt) if np.dtype(dtype).kind == "i" else dt
    rc = fn(nx, ny, ns, _p(dx, dtype), _p(dy, dtype), _p(ds, dtype), T(dt),
            _p(u0, dtype), _p(u1, dtype), _p(v0, dtype), _p(v1, dtype), _p(w0, dtype),
            _p(w1, dtype), C.byref(pc0), C.byref(pc1), 1, order, *extra)
    a0 = C.cast(pc0, C.c_void_p).value
    a1 = C.cast(pc1, C.c_void_p).value
    by_addr = {c0.ctypes.data: c0, c1.ctypes.data: c1}
    return rc, by_addr[a1], by_addr[a0]


def smolar(dx, dy, ds, dt, u0, u1, v0, v1, w0, w1, c0, c1, order, dtype=np.float32,
           **kw):
    """Oracle restatement of smolar(); c0/c1 are modified like the reference's
    buffers.  Returns (rc, newest, other)."""
    lib = oracle_lib()
    fn = getattr(lib, f"oracle_smolar_{_sfx(dtype)}")
    o = opts(**kw)
    return _smolar_call(fn, dtype, dx, dy, ds, dt, u0, u1, v0, v1, w0, w1, c0, c1, order,
                        extra=(C.byref(o),))


def ref_smolar(dx, dy, ds, dt, u0, u1, v0, v1, w0, w1, c0, c1, order, variant="f32"):
    """The reference's own smolar() (compiled from its sources; variant 'i64'
    is its INTEGER build)."""
    lib = ref_lib(variant)
    dtype = {"f64": np.float64, "i64": np.int64}.get(variant, np.float32)
    return _smolar_call(lib.smolar, dtype, dx, dy, ds, dt, u0, u1, v0, v1, w0, w1, c0, c1,
                        order)


def courant(dx, dy, ds, dt, u0, u1, v0, v1, w0, w1, dtype=np.float32):
    ns, ny, nx = u0.shape
    U = np.zeros_like(u0); V = np.zeros_like(u0); W = np.zeros_like(u0)
    fn = getattr(oracle_lib(), f"oracle_courant_{_sfx(dtype)}")
    T = _ct(dtype)
    fn(nx, ny, ns, _p(dx, dtype), _p(dy, dtype), _p(ds, dtype), T(dt), _p(u0, dtype),
       _p(u1, dtype), _p(v0, dtype), _p(v1, dtype), _p(w0, dtype), _p(w1, dtype),
       _p(U, dtype), _p(V, dtype), _p(W, dtype))
    return U, V, W


def step_faces(U, V, W, c0, order, want_inter=False, **kw):
    """One step from advective faces; returns c1 (and the pre-last-pass field)."""
    dtype = c0.dtype
    ns, ny, nx = c0.shape
    c1 = np.zeros_like(c0)
    inter = np.zeros_like(c0) if want_inter else None
    o = opts(**kw)
    fn = getattr(oracle_lib(), f"oracle_step_faces_{_sfx(dtype)}")
    rc = fn(nx, ny, ns, _p(U, dtype), _p(V, dtype), _p(W, dtype), _p(c0, dtype),
            _p(c1, dtype), _p(inter, dtype) if want_inter else None, order, C.byref(o))
    if rc:
        raise RuntimeError(f"oracle step failed: {rc}")
    return (c1, inter) if want_inter else c1


def antidiff(c, Uo, Vo, Wo, Vadv, pass_index, **kw):
    dtype = c.dtype
    ns, ny, nx = c.shape
    Un = np.zeros_like(c); Vn = np.zeros_like(c); Wn = np.zeros_like(c)
    o = opts(**kw)
    fn = getattr(oracle_lib(), f"oracle_antidiff_{_sfx(dtype)}")
    fn(nx, ny, ns, _p(c, dtype), _p(Uo, dtype), _p(Vo, dtype), _p(Wo, dtype),
       _p(Vadv, dtype), pass_index, _p(Un, dtype), _p(Vn, dtype), _p(Wn, dtype), C.byref(o))
    return Un, Vn, Wn


def mass(c) -> float:
    dtype = c.dtype
    ns, ny, nx = c.shape
    fn = getattr(oracle_lib(), f"oracle_mass_{_sfx(dtype)}")
    fn.restype = C.c_double
    return float(fn(nx, ny, ns, _p(c, dtype)))


def ref_test_init(n: int, m: int, variant: str = "f32"):
    """The reference's own test_init(n, m) (tests/init.c:15-103), whose record is
    struct test_config_t (tests/init.h:4-16): returns a dict of numpy copies
    (u, v, w, c0, dx, dy, ds, dt, order, xof, yof)."""
    lib = ref_lib(variant)
    T = C.c_double if variant == "f64" else C.c_float
    dtype = np.float64 if variant == "f64" else np.float32

    class Cfg(C.Structure):
        _fields_ = [("desc", C.c_void_p), ("n", C.c_int), ("m", C.c_int), ("dt", T),
                    ("u", C.POINTER(T)), ("v", C.POINTER(T)), ("w", C.POINTER(T)),
                    ("c0", C.POINTER(T)), ("c1", C.POINTER(T)), ("dx", C.POINTER(T)),
                    ("dy", C.POINTER(T)), ("ds", C.POINTER(T)), ("order", C.c_int),
                    ("flow_type", C.c_int), ("xof", C.c_int), ("yof", C.c_int)]

    lib.test_init.restype = C.POINTER(Cfg)
    size = C.c_int(0)
    cfg = lib.test_init(n, m, C.byref(size)).contents
    npts = n * n * m

    def grab(ptr, count):
        return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dtype).copy()

    out = dict(
        u=grab(cfg.u, npts).reshape(m, n, n), v=grab(cfg.v, npts).reshape(m, n, n),
        w=grab(cfg.w, npts).reshape(m, n, n), c0=grab(cfg.c0, npts).reshape(m, n, n),
        dx=grab(cfg.dx, n), dy=grab(cfg.dy, n), ds=grab(cfg.ds, m), dt=float(cfg.dt),
        order=cfg.order, xof=cfg.xof, yof=cfg.yof)
    libc = C.CDLL(None)
    libc.free(C.c_void_p(C.addressof(cfg)))
    return out
