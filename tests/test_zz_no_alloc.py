"""GPU test of mpdata_step_noalloc(), the entry point for callers that cannot
allocate device memory while they run (stream capture, fixed memory budgets,
host frameworks owning the allocator).

It is called through the C ABI with device pointers, twice in a row (the
second call stepping the first call's output), and both results are compared
with the regular handle API (mpdata_create/mpdata_step) within the float32
tolerance the other GPU tests use (max abs difference <= 1e-5).  The file is
named to be collected last, so a run stopping at the first failure has run
every other test already; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _faces_and_field(nx, ny, ns, seed):
    import oracle
    from mpdata_b200 import workloads
    case = workloads.random_case(nx, ny, ns, seed=seed)
    U, V, W = oracle.courant(case["dx"], case["dy"], case["ds"], case["dt"], case["u0"],
                             case["u1"], case["v0"], case["v1"], case["w0"], case["w1"],
                             dtype=np.float64)
    return [x.astype(np.float32) for x in (U, V, W)], case["c0"].astype(np.float32)


@pytest.mark.parametrize("limiter", [0, 1])
@pytest.mark.parametrize("order", [1, 2, 3])
def test_noalloc_step_matches_handle_api_twice(limiter, order):
    import torch

    import mpdata_b200 as m

    nx, ny, ns = 53, 37, 19
    (U, V, W), c0 = _faces_and_field(nx, ny, ns, seed=order + 5 * limiter)
    dev = torch.device("cuda", 0)
    dU, dV, dW = (torch.from_numpy(x).to(dev) for x in (U, V, W))
    a = torch.from_numpy(c0).to(dev)
    b = torch.empty_like(a)
    c = torch.empty_like(a)
    stream = torch.cuda.current_stream()
    fn = m.library().mpdata_step_noalloc
    fn.argtypes = [C.c_int] * 5 + [C.c_void_p] * 5 + [C.c_void_p]
    ptr = lambda t: C.c_void_p(t.data_ptr())
    outs = []
    for src, dst in ((a, b), (b, c)):
        rc = fn(nx, ny, ns, order, limiter, ptr(dU), ptr(dV), ptr(dW), ptr(src), ptr(dst),
                C.c_void_p(stream.cuda_stream))
        assert rc == 0, m.last_error()
        stream.synchronize()
        outs.append(dst.cpu().numpy().copy())

    with m.Solver(nx, ny, ns, order=order, limiter=bool(limiter)) as s:
        s.set_faces(U, V, W)
        s.set_field(c0)
        for got in outs:
            s.step(1)
            ref = s.get_field()
            assert np.abs(got - ref).max() <= TOL


def test_noalloc_rejects_grids_beyond_the_static_scratch():
    import mpdata_b200 as m
    fn = m.library().mpdata_step_noalloc
    fn.argtypes = [C.c_int] * 5 + [C.c_void_p] * 5 + [C.c_void_p]
    one = C.c_void_p(16)  # never dereferenced: the size check comes first
    other = C.c_void_p(32)
    rc = fn(512, 512, 256, 2, 0, one, one, one, one, other, None)
    assert rc == -1
    assert "static scratch" in m.last_error()
