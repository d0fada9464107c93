"""The throughput workload at its full size (512 x 512 x 256 FP32, IORD 3 +
limiter, streamfunction flow): properties that do not depend on the size.

* the headline arithmetic (two-cell pass, limiter, approx_div) leaves no
  negative cell and stays within relative L2 1e-5 of an FP64 run of the
  plain method after 10 steps;
* with the y faces of the x = 1 column computed (vv_fix, the benchmark's
  setting), every FP32 form stays within relative L2 1e-5 of the FP64 run
  over the configuration's 100 steps;
* a z-chunked march gives the same bits as the whole-column one at every
  chunk depth (chunks of 96 planes are the default here);
* a grid of more than 2^31 elements per field steps correctly (64-bit
  offsets throughout).
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


@pytest.mark.parametrize("form", [dict(approx_div=True), dict(approx_div=True, precision_form=True),
                                  dict()], ids=["approx_div", "precision_form", "plain"])
def test_fullsize_100_steps_within_fp64_bound(m, wl, form):
    """The throughput configuration over its own length (100 steps) with the
    y faces of the x = 1 column computed (vv_fix): every FP32 form within
    relative L2 1e-5 of the FP64 run, no negative cell."""
    c64, _, _ = _steps(m, wl, 100, dtype=np.float64, vv_fix=True)
    c32, mn, nneg = _steps(m, wl, 100, vv_fix=True, **form)
    rel = np.linalg.norm(c32.astype(np.float64) - c64) / np.linalg.norm(c64)
    assert rel <= REL_L2_BOUND, rel
    assert nneg == 0 and mn >= 0.0


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


def test_grid_beyond_32bit_offsets(m):
    """1024 x 1024 x 2049 cells (2.15e9 > 2^31 elements per field, ~105 GB of
    solver state): a problem that is one-dimensional in z (U = V = 0,
    constant W, a field varying in z only) gives every interior column the
    same arithmetic, so each column -- the far corner's too, whose offsets
    need 64 bits -- must equal the column of a 6 x 6 x 2049 grid bit for bit."""
    torch = pytest.importorskip("torch")
    torch.cuda.empty_cache()
    free, _ = torch.cuda.mem_get_info()
    if free < 130e9:  # 103 GB of solver state + 17 GB of inputs at the peak
        pytest.skip(f"needs 130 GB of free device memory, {free / 1e9:.0f} GB free")
    ns = 2049
    z = torch.linspace(0.0, 12.0, ns, dtype=torch.float64)
    prof = (1.0 + torch.sin(z) * torch.exp(-0.05 * z)).to(torch.float32).cuda()

    def run(nx, ny):
        s = m.Solver(nx, ny, ns, order=2, kernel=3)  # the two-cell pass at both sizes
        try:
            # device arrays are read on the handle's stream: share torch's, so
            # the copies follow the fills and precede the reuse of freed blocks
            s.set_stream(torch.cuda.current_stream().cuda_stream)
            shape = (ns, ny, nx)
            zero = torch.zeros(shape, dtype=torch.float32, device="cuda")
            W = torch.full(shape, 0.3, dtype=torch.float32, device="cuda")
            s.set_faces(zero, zero, W)
            del W
            c = prof.view(ns, 1, 1).expand(shape).contiguous()
            s.set_field(c)
            del c, zero
            torch.cuda.empty_cache()
            s.step(2)
            out = torch.empty(shape, dtype=torch.float32, device="cuda")
            s.get_field(out)
            s.sync()
            cols = [out[:, 1, 1].clone(), out[:, ny // 2, nx // 2].clone(),
                    out[:, ny - 2, nx - 2].clone()]
            del out
            torch.cuda.empty_cache()
            return cols
        finally:
            s.close()

    small = run(6, 6)
    big = run(1024, 1024)
    for col in big + small[1:]:
        assert torch.equal(col, small[0])
    assert not torch.equal(small[0], prof)  # the step moved the profile
