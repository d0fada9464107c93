"""Velocity updates through the handle API (mpdata_set_velocity).

The advective faces of a velocity update are formed by the next step's
pass 0, in one march with the donor update (k_courant_donor_v), instead of
by a separate Courant kernel whose output pass 0 reads back.  The faces and
the field must be the same bits as the separate kernels give (the Courant
check still forms the faces at once, so it serves as the comparison), equal
to the oracle in strict mode, and a later velocity update or set_faces must
supersede a pending one.  Inputs: two time levels (u0 != u1) and
non-uniform grid steps.
"""
import numpy as np
import pytest

from mpdata_b200 import workloads

pytestmark = pytest.mark.gpu

NX, NY, NS = 37, 23, 19


@pytest.fixture(scope="module")
def m():
    import mpdata_b200
    return mpdata_b200


def _case(seed, dtype=np.float32):
    g = workloads.random_case(NX, NY, NS, seed=seed)
    return {k: (v.astype(dtype) if isinstance(v, np.ndarray) else v) for k, v in g.items()}


def _vel(f):
    return (f["dx"], f["dy"], f["ds"], f["dt"], f["u0"], f["u1"], f["v0"], f["v1"], f["w0"], f["w1"])


def _run(m, f, order, steps, dtype=np.float32, **opts):
    s = m.Solver(NX, NY, NS, order=order, dtype=dtype, **opts)
    try:
        s.set_velocity(*_vel(f))
        s.set_field(f["c0"])
        s.step(steps)
        return s.get_field(), s.get_field(previous=True)
    finally:
        s.close()


@pytest.mark.parametrize("dtype", [np.float32, np.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("opts", [dict(), dict(limiter=True), dict(strict=True),
                                  dict(limiter=True, strict=True)],
                         ids=["plain", "limiter", "strict", "strict-limiter"])
def test_faces_in_pass0_same_bits_as_separate_kernels(m, dtype, order, opts):
    f = _case(order + 11, dtype)
    fused = _run(m, f, order, 3, dtype, **opts)
    eager = _run(m, f, order, 3, dtype, check_courant=True, **opts)  # faces formed at once
    assert np.array_equal(fused[0], eager[0]) and np.array_equal(fused[1], eager[1])


@pytest.mark.parametrize("order", [1, 2, 3])
def test_faces_in_pass0_strict_equals_oracle(m, oracle_mod, order):
    f = _case(order + 29, np.float64)
    got, _ = _run(m, f, order, 2, np.float64, strict=True)
    c0, c1 = f["c0"].copy(), np.zeros_like(f["c0"])
    for _ in range(2):  # the oracle recomputes the faces per call, as the reference does
        rc, newest, other = oracle_mod.smolar(*_vel(f), c0, c1, order, dtype=np.float64)
        assert rc == 0
        c0, c1 = newest.copy(), other.copy()
    assert np.array_equal(got, c0)


@pytest.mark.parametrize("dtype", [np.float32, np.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("order", [1, 3])
@pytest.mark.parametrize("opts", [dict(), dict(limiter=True, approx_div=True), dict(strict=True)],
                         ids=["plain", "limiter-approx", "strict"])
def test_one_level_velocities_same_bits(m, dtype, order, opts):
    """One array per component for both time levels (as the reference's
    drivers pass them): the fused march loads each once; faces and field are
    the bits of the separate kernels."""
    if dtype == np.float64 and opts.get("approx_div"):
        pytest.skip("approx_div is a float32 form")
    f = _case(order + 51, dtype)
    f["u1"], f["v1"], f["w1"] = f["u0"], f["v0"], f["w0"]
    fused = _run(m, f, order, 3, dtype, **opts)
    eager = _run(m, f, order, 3, dtype, check_courant=True, **opts)
    assert np.array_equal(fused[0], eager[0]) and np.array_equal(fused[1], eager[1])


def test_later_update_supersedes_pending_one(m):
    a, b = _case(41), _case(42)
    s = m.Solver(NX, NY, NS, order=2, limiter=True)
    try:
        s.set_velocity(*_vel(a))
        s.set_velocity(*_vel(b))  # before any step: only b's faces may count
        s.set_field(b["c0"])
        s.step(2)
        got = s.get_field()
    finally:
        s.close()
    assert np.array_equal(got, _run(m, b, 2, 2, limiter=True)[0])


def test_set_faces_supersedes_pending_update(m):
    a, b = _case(43), _case(44)
    U, V, W = workloads.faces_from_cells(b["u0"], b["v0"], b["w0"])
    faces = [np.ascontiguousarray(x, np.float32) for x in (U, V, W)]
    s = m.Solver(NX, NY, NS, order=2)
    t = m.Solver(NX, NY, NS, order=2)
    try:
        s.set_velocity(*_vel(a))
        s.set_faces(*faces)  # replaces the pending update
        t.set_faces(*faces)
        for x in (s, t):
            x.set_field(b["c0"])
            x.step(2)
        assert np.array_equal(s.get_field(), t.get_field())
    finally:
        s.close()
        t.close()


@pytest.mark.parametrize("nx", [64, NX], ids=["in-place", "copied"])  # px == nx only for 64
def test_lent_device_arrays_same_bits_as_copied(m, nx):
    """MPDATA_DEVICE_BORROW: the step reads the caller's device arrays in place
    (rows of pitch nx, a multiple of 32) or, for another layout, copies them;
    either way the bits equal those of a copied update.  The lent arrays are
    overwritten after the step has run: later steps do not read them."""
    torch = pytest.importorskip("torch")
    g = workloads.random_case(nx, NY, NS, seed=nx + 5)
    f = {k: (v.astype(np.float32) if isinstance(v, np.ndarray) else v) for k, v in g.items()}
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray) else v
           for k, v in f.items()}
    out = []
    for borrow in (False, True):
        s = m.Solver(nx, NY, NS, order=3, limiter=True, approx_div=True)
        try:
            s.set_stream(torch.cuda.current_stream().cuda_stream)
            vel = [dev[k].clone() if isinstance(dev[k], torch.Tensor) else dev[k] for k in
                   ("dx", "dy", "ds", "dt", "u0", "u1", "v0", "v1", "w0", "w1")]
            s.set_velocity(*vel, borrow=borrow)
            s.set_field(f["c0"])
            s.step(1)
            s.sync()
            for t in vel:
                if isinstance(t, torch.Tensor):
                    t.fill_(7.0)  # the update has been consumed
            s.step(2)
            out.append(s.get_field())
        finally:
            s.close()
    assert np.array_equal(out[0], out[1])


def test_borrow_is_for_velocities_only(m):
    """The other copy entry points reject MPDATA_DEVICE_BORROW (MPDATA_ERR_ARG)."""
    import ctypes as C
    torch = pytest.importorskip("torch")
    s = m.Solver(NX, NY, NS, order=2)
    try:
        c = torch.zeros((NS, NY, NX), dtype=torch.float32, device="cuda")
        p = C.c_void_p(c.data_ptr())
        lib = m.library()
        assert lib.mpdata_set_field(s._h, p, m.DEVICE_BORROW) == -1
        assert lib.mpdata_set_faces(s._h, p, p, p, m.DEVICE_BORROW) == -1
        assert lib.mpdata_set_field(s._h, p, m.DEVICE) == 0
        assert lib.mpdata_get_field(s._h, p, m.DEVICE_BORROW) == -1
        assert lib.mpdata_get_planes(s._h, 0, 1, p, m.DEVICE_BORROW) == -1
        assert lib.mpdata_set_planes(s._h, 0, 1, p, m.DEVICE_BORROW) == -1
    finally:
        s.close()
