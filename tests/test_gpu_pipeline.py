"""The pipelined host step of smolar() (mpdata_set_pipeline).

smolar() uploads velocities and field and downloads two fields on every
call; the pipelined form overlaps those copies and the kernels chunk by
chunk of z planes.  It runs the same kernels on the same planes, so its
outputs must be the same bits as the unpipelined step's, for every chunk
size, order, precision and option, over several driver-style calls (the
newest output becomes the next input), with pageable and pinned host
buffers.
"""
import ctypes as C

import numpy as np
import pytest

from mpdata_b200 import workloads

pytestmark = pytest.mark.gpu

NX, NY, NS = 37, 21, 40


@pytest.fixture(scope="module")
def m():
    import mpdata_b200
    yield mpdata_b200
    mpdata_b200.set_pipeline(0)
    mpdata_b200.set_default_options(None)


def _run(m, f, order, chunk, steps, dtype, buffers=None):
    m.set_pipeline(chunk)
    c0 = f["c0"].astype(dtype).copy() if buffers is None else buffers[0]
    c1 = np.zeros_like(c0) if buffers is None else buffers[1]
    if buffers is not None:
        c0[...] = f["c0"]
        c1[...] = 0
    outs = []
    for _ in range(steps):
        a, b = m.smolar(NX, NY, NS, f["dx"], f["dy"], f["ds"], f["dt"], f["u0"], f["u1"],
                        f["v0"], f["v1"], f["w0"], f["w1"], c0, c1, order=order, dtype=dtype)
        outs.append((a.copy(), b.copy()))
        c0, c1 = b, a  # driver exchange: the newest field is the next input
    return outs


@pytest.mark.parametrize("dtype", [np.float32, np.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("order", [1, 2, 3, 4])
@pytest.mark.parametrize("opt", [dict(), dict(limiter=True), dict(limiter=True, strict=True),
                                 dict(limiter=True, approx_div=True)],
                         ids=["plain", "limiter", "strict", "approx"])
def test_pipelined_smolar_same_bits(m, dtype, order, opt):
    if opt.get("approx_div") and dtype is np.float64:
        pytest.skip("approx_div is an FP32 form")
    g = workloads.random_case(NX, NY, NS, seed=order + 3)
    f = {k: (v.astype(dtype) if isinstance(v, np.ndarray) else v) for k, v in g.items()}
    m.set_default_options(m.SolverOptions(**opt))
    try:
        ref = _run(m, f, order, -1, 3, dtype)
        for chunk in (4, 5, 7, 13, 17, 0):
            got = _run(m, f, order, chunk, 3, dtype)
            for (ga, gb), (ra, rb) in zip(got, ref):
                assert np.array_equal(ga, ra) and np.array_equal(gb, rb), chunk
    finally:
        m.set_default_options(None)


def test_queued_plane_copies_overlap_steps(m):
    """mpdata_get_planes(MPDATA_HOST_ASYNC) + mpdata_wait: step k+1 and its
    plane copy are queued before the planes of step k are read (the ring
    driver's frame output); every frame equals the synchronous copy of a
    solver stepped alongside."""
    g = workloads.random_case(NX, NY, NS, seed=23)
    f = {k: (v.astype(np.float32) if isinstance(v, np.ndarray) else v) for k, v in g.items()}
    args = (f["dx"], f["dy"], f["ds"], f["dt"], f["u0"], f["u1"], f["v0"], f["v1"], f["w0"],
            f["w1"])
    q, r = (m.Solver(NX, NY, NS, order=3, limiter=True) for _ in range(2))
    for s in (q, r):
        s.set_velocity(*args)
        s.set_field(f["c0"])
    lib = m.library()
    nb = 2 * NY * NX
    ptrs = [lib.mpdata_host_alloc(4 * nb) for _ in range(2)]
    try:
        buf = [np.ctypeslib.as_array((C.c_float * nb).from_address(p)).reshape(2, NY, NX)
               for p in ptrs]
        steps, tk = 6, [None, None]
        q.step(1)
        tk[1] = q.get_planes_async(1, 2, buf[1])
        for it in range(1, steps + 1):
            b = it & 1
            if it < steps:
                q.step(1)
                tk[b ^ 1] = q.get_planes_async(1, 2, buf[b ^ 1])
            q.wait(tk[b])
            r.step(1)
            assert np.array_equal(buf[b], r.get_planes(1, 2)), it
        with pytest.raises(m.MpdataError):
            q.wait(-1)
        # an unknown destination kind is an argument error, not a copy
        out = np.zeros((2, NY, NX), np.float32)
        rc = m.library().mpdata_get_planes(q._h, 1, 2, C.c_void_p(out.ctypes.data), 7)
        assert rc == -1 and not out.any()
    finally:
        q.close()
        r.close()
        for p in ptrs:
            lib.mpdata_host_free(C.c_void_p(p))


def test_pipelined_smolar_pinned_buffers(m):
    """Pinned host buffers (every copy asynchronous) give the same bits."""
    g = workloads.random_case(NX, NY, NS, seed=17)
    f = {k: (v.astype(np.float32) if isinstance(v, np.ndarray) else v) for k, v in g.items()}
    lib = m.library()
    n = NX * NY * NS
    ptrs = [lib.mpdata_host_alloc(4 * n) for _ in range(2)]
    try:
        bufs = [np.ctypeslib.as_array((C.c_float * n).from_address(p)).reshape(NS, NY, NX)
                for p in ptrs]
        m.set_default_options(m.SolverOptions(limiter=True, approx_div=True))
        ref = _run(m, f, 3, -1, 3, np.float32)
        got = _run(m, f, 3, 6, 3, np.float32, buffers=bufs)
        for (ga, gb), (ra, rb) in zip(got, ref):
            assert np.array_equal(ga, ra) and np.array_equal(gb, rb)
    finally:
        m.set_default_options(None)
        for p in ptrs:
            lib.mpdata_host_free(C.c_void_p(p))
