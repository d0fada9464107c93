"""Adjoint of a window of MPDATA steps (``mpdata_adjoint_*`` C ABI) and a
``torch.autograd.Function`` wrapper used as a gradient-check harness.

The C library does all the work: the forward window (with checkpoints every
``checkpoint_every`` steps) and the hand-written reverse kernels.  torch is
used only for device buffers and to chain the window into autograd graphs
(receptor losses, source amplitudes) in the tests.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import (DEVICE, HOST, Options, SolverOptions, _check, _dtype_code, _lib, _ptr)

_vp = C.c_void_p
_lib.mpdata_adjoint_create.argtypes = [C.POINTER(_vp), C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_int, C.POINTER(Options), C.c_int]
_lib.mpdata_adjoint_destroy.argtypes = [_vp]
_lib.mpdata_adjoint_set_stream.argtypes = [_vp, _vp]
_lib.mpdata_adjoint_set_faces.argtypes = [_vp, _vp, _vp, _vp, C.c_int]
_lib.mpdata_adjoint_forward.argtypes = [_vp, _vp, C.c_int, _vp, C.c_int]
_lib.mpdata_adjoint_backward.argtypes = [_vp, _vp, _vp, C.c_int]


class Adjoint:
    """Forward window + reverse sweep with step checkpointing."""

    def __init__(self, nx, ny, ns, order=2, dtype=np.float32, checkpoint_every=20,
                 options: SolverOptions | None = None, **kw):
        opts = options or SolverOptions(**kw)
        self.shape = (ns, ny, nx)
        self.dtype = np.dtype(dtype)
        self._h = C.c_void_p(None)
        o = opts.to_c()
        _check(_lib.mpdata_adjoint_create(C.byref(self._h), nx, ny, ns, _dtype_code(dtype), order,
                                          C.byref(o), checkpoint_every))

    def close(self):
        if self._h and self._h.value:
            _lib.mpdata_adjoint_destroy(self._h)
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
        _check(_lib.mpdata_adjoint_set_stream(self._h, C.c_void_p(stream_handle)))

    def set_faces(self, U, V, W):
        p = [_ptr(x, self.dtype) for x in (U, V, W)]
        _check(_lib.mpdata_adjoint_set_faces(self._h, p[0][0], p[1][0], p[2][0], p[0][1]))

    def forward(self, c0, nsteps, out=None):
        """Run the window; returns c^N (numpy for a numpy input)."""
        p0, where = _ptr(c0, self.dtype)
        if out is None and where == HOST:
            out = np.empty(self.shape, self.dtype)
        pn = _ptr(out, self.dtype)[0] if out is not None else None
        _check(_lib.mpdata_adjoint_forward(self._h, p0, nsteps, pn, where))
        return out

    def backward(self, lamN, out=None):
        """Adjoint of the last window: lamN (d loss / d c^N) -> d loss / d c^0."""
        pl, where = _ptr(lamN, self.dtype)
        if out is None:
            if where == HOST:
                out = np.empty(self.shape, self.dtype)
            else:
                import torch
                out = torch.empty_like(lamN)
        _check(_lib.mpdata_adjoint_backward(self._h, pl, _ptr(out, self.dtype)[0], where))
        return out


def window_function():
    """torch.autograd.Function running an :class:`Adjoint` window:
    ``MpdataWindow.apply(c0, adjoint, nsteps)`` -> c^N, differentiable in c0
    (CUDA tensors)."""
    import torch

    class MpdataWindow(torch.autograd.Function):
        @staticmethod
        def forward(ctx, c0, adjoint: Adjoint, nsteps: int):
            c0 = c0.contiguous()
            torch.cuda.current_stream().synchronize()
            cN = torch.empty_like(c0)
            adjoint.forward(c0, nsteps, out=cN)
            ctx.adjoint = adjoint
            return cN

        @staticmethod
        def backward(ctx, gN):
            torch.cuda.current_stream().synchronize()
            g0 = ctx.adjoint.backward(gN.contiguous())
            return g0, None, None

    return MpdataWindow


__all__ = ["Adjoint", "window_function", "DEVICE", "HOST"]
