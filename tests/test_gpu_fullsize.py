"""The throughput workload at its full size (512 x 512 x 256 FP32, IORD 3 +
limiter, streamfunction flow): properties that do not depend on the size.

* the headline arithmetic (two-cell pass, limiter, approx_div) leaves no
  negative cell and stays within relative L2 1e-5 of an FP64 run of the
  plain method after 10 steps;
* a z-chunked march gives the same bits as the whole-column one at every
  chunk depth (chunks of 96 planes are the default here).
"""
import numpy as np
import pytest

from mpdata_b200 import workloads

pytestmark = pytest.mark.gpu

NX, NY, NS, ORDER = 512, 512, 256, 3
REL_L2_BOUND = 1e-5


@pytest.fixture(scope="module")
def m():
    import mpdata_b200
    return mpdata_b200


@pytest.fixture(scope="module")
def wl():
    return workloads.roofline(NX, NY, NS)


def _steps(m, wl, steps, dtype=np.float32, depth=None, **opts):
    s = m.Solver(NX, NY, NS, order=ORDER, dtype=dtype, limiter=True, **opts)
    try:
        s.set_faces(*(np.ascontiguousarray(wl[k], dtype) for k in ("U", "V", "W")))
        s.set_field(np.ascontiguousarray(wl["c0"], dtype))
        if depth is not None:
            s.set_march_depth(depth)
        s.step(steps)
        mn, nneg = s.min()
        return s.get_field(), mn, nneg
    finally:
        s.close()


def test_fullsize_positive_and_close_to_fp64(m, wl):
    c32, mn, nneg = _steps(m, wl, 10, approx_div=True)
    assert nneg == 0 and mn >= 0.0
    c64, _, _ = _steps(m, wl, 10, dtype=np.float64)
    rel = np.linalg.norm(c32.astype(np.float64) - c64) / np.linalg.norm(c64)
    assert rel <= REL_L2_BOUND, rel


@pytest.mark.parametrize("opts", [dict(approx_div=True), dict()], ids=["approx", "ieee"])
def test_fullsize_chunked_march_same_bits(m, wl, opts):
    ref, _, _ = _steps(m, wl, 3, depth=0, **opts)
    for depth in (None, 32):
        got, _, _ = _steps(m, wl, 3, depth=depth, **opts)
        assert np.array_equal(got, ref), depth
