"""GPU parity: the CUDA path against the CPU oracle and the reference's own
outputs, through the C ABI.

Tolerances (stated here, checked below):
  strict mode (-fmad=false kernels)      bit-identical to the oracle / fixtures
  default mode, float32                  max |gpu - oracle| <= 1e-5 (fields O(1))
  default mode, float64                  max |gpu - oracle| <= 1e-11
  FP32 storage form vs FP64 plain run    relative L2 <= 1e-5
"""
import os

import numpy as np
import pytest

from conftest import golden_files, load_golden
from mpdata_b200 import workloads

pytestmark = pytest.mark.gpu

TOL = {np.dtype(np.float32): 1e-5, np.dtype(np.float64): 1e-11}


@pytest.fixture(scope="module")
def m():
    import mpdata_b200
    yield mpdata_b200
    mpdata_b200.set_default_options(None)


def _smolar_steps(m, g, dtype, steps):
    c0 = g["c0"].astype(dtype).copy()
    c1 = np.zeros_like(c0)
    for _ in range(steps):
        a, b = m.smolar(c0.shape[2], c0.shape[1], c0.shape[0], g["dx"].astype(dtype),
                        g["dy"].astype(dtype), g["ds"].astype(dtype), float(g["dt"]),
                        *(g[k].astype(dtype) for k in ("u0", "u1", "v0", "v1", "w0", "w1")),
                        c0, c1, order=int(g["order"]), dtype=dtype)
        c0, c1 = b.copy(), a.copy()  # driver exchange: newest becomes the input
    return c0, c1


@pytest.mark.parametrize("kernel", [0, 1], ids=["fused", "unfused"])
@pytest.mark.parametrize("path", golden_files(floating_only=True), ids=os.path.basename)
def test_smolar_strict_reproduces_reference_fixtures(m, path, kernel):
    g = load_golden(path)
    m.set_default_options(m.SolverOptions(strict=True, kernel=kernel))
    newest, other = _smolar_steps(m, g, g["c0"].dtype, int(g["steps"]))
    assert np.array_equal(newest, g["newest"])
    assert np.array_equal(other, g["other"])


@pytest.mark.parametrize("path", golden_files(floating_only=True), ids=os.path.basename)
def test_smolar_default_within_tolerance(m, path):
    g = load_golden(path)
    m.set_default_options(None)
    newest, _ = _smolar_steps(m, g, g["c0"].dtype, int(g["steps"]))
    assert np.abs(newest - g["newest"]).max() <= TOL[g["c0"].dtype]


def test_smolar_pointer_exchange_matches_reference(m):
    g = workloads.random_case(9, 8, 7, seed=5)
    f = {k: (v.astype(np.float32) if isinstance(v, np.ndarray) else v) for k, v in g.items()}
    m.set_default_options(None)
    for order in (1, 2, 3, 4):
        c0 = f["c0"].copy(); c1 = np.zeros_like(c0)
        a, b = m.smolar(9, 8, 7, f["dx"], f["dy"], f["ds"], f["dt"], f["u0"], f["u1"], f["v0"],
                        f["v1"], f["w0"], f["w1"], c0, c1, order=order)
        swapped = a is c1
        assert swapped == (order % 2 == 0)


def _faces(case, dtype):
    import oracle
    U, V, W = oracle.courant(case["dx"], case["dy"], case["ds"], case["dt"], case["u0"],
                             case["u1"], case["v0"], case["v1"], case["w0"], case["w1"],
                             dtype=np.float64)
    return U.astype(dtype), V.astype(dtype), W.astype(dtype)


SHAPES = [(70, 21, 9), (35, 12, 5), (130, 19, 4), (33, 9, 3), (3, 3, 3), (40, 40, 40)]
OPTS = [dict(), dict(limiter=1), dict(vv_fix=1), dict(div_mode=1), dict(limiter=1, vv_fix=1)]


@pytest.mark.parametrize("kernel", [0, 1], ids=["fused", "unfused"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("order", [1, 2, 3, 4])
@pytest.mark.parametrize("opt", OPTS, ids=lambda o: "-".join(o) or "plain")
def test_handle_strict_bit_exact(m, kernel, dtype, shape, order, opt):
    import oracle
    nx, ny, ns = shape
    case = workloads.random_case(nx, ny, ns, seed=nx + ny + ns + order)
    U, V, W = _faces(case, dtype)
    c = case["c0"].astype(dtype)
    ref = c
    for _ in range(2):
        ref = oracle.step_faces(U, V, W, ref, order, **opt)
    with m.Solver(nx, ny, ns, order=order, dtype=dtype, strict=True, kernel=kernel,
                  limiter=bool(opt.get("limiter")), vv_fix=bool(opt.get("vv_fix")),
                  div_mode=opt.get("div_mode", 0)) as s:
        s.set_faces(U, V, W)
        s.set_field(c)
        s.step(2)
        got = s.get_field()
    assert np.array_equal(got, ref), np.abs(got - ref).max()


@pytest.mark.parametrize("depth", [1, 2, 5, 13, 0])
@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("limiter", [0, 1])
def test_z_chunked_march_strict_bit_exact(m, depth, order, limiter):
    """Chunking the z march (any depth, chunk edges anywhere) changes nothing."""
    import oracle
    nx, ny, ns = 37, 21, 30
    case = workloads.random_case(nx, ny, ns, seed=depth + 7 * order)
    U, V, W = _faces(case, np.float32)
    c = case["c0"].astype(np.float32)
    ref = c
    for _ in range(2):
        ref = oracle.step_faces(U, V, W, ref, order, limiter=limiter)
    with m.Solver(nx, ny, ns, order=order, strict=True, limiter=bool(limiter)) as s:
        s.set_march_depth(depth)
        s.set_faces(U, V, W)
        s.set_field(c)
        s.step(2)
        assert np.array_equal(s.get_field(), ref)


def test_autotune_keeps_field_and_results():
    import oracle
    nx, ny, ns = 66, 34, 40
    case = workloads.random_case(nx, ny, ns, seed=21)
    U, V, W = _faces(case, np.float32)
    c = case["c0"].astype(np.float32)
    ref = oracle.step_faces(U, V, W, c, 3, limiter=1)
    with m_solver(nx, ny, ns) as s:
        s.set_faces(U, V, W)
        s.set_field(c)
        depth, ms = s.autotune(trial_steps=2)
        assert ms > 0 and depth in (0, 128, 64, 32, 16, 8)
        assert np.array_equal(s.get_field(), c)
        s.step(1)
        assert np.array_equal(s.get_field(), ref)


def m_solver(nx, ny, ns):
    import mpdata_b200
    return mpdata_b200.Solver(nx, ny, ns, order=3, strict=True, limiter=True)


@pytest.mark.parametrize("kernel", [0, 1], ids=["fused", "unfused"])
@pytest.mark.parametrize("order", [2, 3])
def test_precision_form_strict_bit_exact(m, kernel, order):
    import oracle
    case = workloads.random_case(45, 17, 10, seed=order)
    U, V, W = _faces(case, np.float32)
    c = case["c0"].astype(np.float32)
    ref = oracle.step_faces(U, V, W, c, order, limiter=1, wide_beta=1)
    with m.Solver(45, 17, 10, order=order, strict=True, kernel=kernel, limiter=True,
                  precision_form=True) as s:
        s.set_faces(U, V, W)
        s.set_field(c)
        s.step(1)
        assert np.array_equal(s.get_field(), ref)


@pytest.mark.parametrize("dtype", [np.float32, np.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("limiter", [0, 1])
def test_handle_default_mode_within_tolerance(m, dtype, limiter):
    import oracle
    case = workloads.random_case(66, 30, 12, seed=11)
    U, V, W = _faces(case, dtype)
    c = case["c0"].astype(dtype)
    ref = c
    for _ in range(5):
        ref = oracle.step_faces(U, V, W, ref, 3, limiter=limiter)
    with m.Solver(66, 30, 12, order=3, dtype=dtype, limiter=bool(limiter)) as s:
        s.set_faces(U, V, W)
        s.set_field(c)
        s.step(5)
        got = s.get_field()
    assert np.abs(got - ref).max() <= TOL[np.dtype(dtype)]


@pytest.mark.parametrize("limiter", [0, 1])
@pytest.mark.parametrize("precision_form", [0, 1])
def test_approx_div_within_tolerance(m, limiter, precision_form):
    """Hardware-reciprocal ratios (approx_div): FP32 max-abs <= 1e-5 against
    the IEEE oracle after 5 steps of IORD 3."""
    import oracle
    if precision_form and not limiter:
        pytest.skip("the precision form only changes the limiter")
    case = workloads.random_case(66, 30, 12, seed=12)
    U, V, W = _faces(case, np.float32)
    c = case["c0"].astype(np.float32)
    ref = c
    for _ in range(5):
        ref = oracle.step_faces(U, V, W, ref, 3, limiter=limiter, wide_beta=precision_form)
    with m.Solver(66, 30, 12, order=3, limiter=bool(limiter), approx_div=True,
                  precision_form=bool(precision_form)) as s:
        s.set_faces(U, V, W)
        s.set_field(c)
        s.step(5)
        got = s.get_field()
    assert np.abs(got - ref).max() <= TOL[np.dtype(np.float32)]


def test_previous_level_matches_oracle(m):
    import oracle
    case = workloads.random_case(37, 11, 6, seed=2)
    U, V, W = _faces(case, np.float64)
    c = case["c0"]
    newest, inter = oracle.step_faces(U, V, W, c, 3, want_inter=True)
    with m.Solver(37, 11, 6, order=3, dtype=np.float64, strict=True) as s:
        s.set_faces(U, V, W)
        s.set_field(c)
        s.step(1)
        assert np.array_equal(s.get_field(), newest)
        assert np.array_equal(s.get_field(previous=True), inter)


@pytest.mark.parametrize("split", [(2, 2, 1), (3, 1, 2), (4, 3, 2), (1, 1, 1), (40, 1, 1)])
@pytest.mark.parametrize("order", [1, 2, 3])
def test_msmolar_equals_smolar(m, split, order):
    """The decomposed step reproduces the single-domain step bit for bit (the
    reference's intent; its own 1-cell halo misses it by up to 0.2)."""
    m.set_default_options(None)
    nx, ny, ns = 40, 23, 11
    case = workloads.random_case(nx, ny, ns, seed=order)
    f = {k: (v.astype(np.float32) if isinstance(v, np.ndarray) else v) for k, v in case.items()}
    vel = (f["u0"], f["u1"], f["v0"], f["v1"], f["w0"], f["w1"])
    a0 = f["c0"].copy(); a1 = np.zeros_like(a0)
    st = m.MsmolarState()
    b0 = f["c0"].copy(); b1 = np.zeros_like(b0)
    for _ in range(3):
        a0, a1 = m.smolar(nx, ny, ns, f["dx"], f["dy"], f["ds"], f["dt"], *vel, a0, a1,
                          order=order)
        a0, a1 = a1, a0  # driver exchange
        b0, b1 = m.msmolar(st, nx, ny, ns, f["dx"], f["dy"], f["ds"], f["dt"], *vel, b0, b1,
                           order=order, sx=split[0], sy=split[1], ss=split[2])
        b0, b1 = b1, b0
    # after the driver exchange the newest sits in *c0; gather fills *c1/*c0
    g0, g1 = m.msmolar_gather(st, nx, ny, ns, f["dx"], f["dy"], f["ds"], f["dt"], *vel, b1,
                              b0, order=order, sx=split[0], sy=split[1], ss=split[2])
    st.free()
    assert np.array_equal(g1, a0)


def test_ring2d_reference_form_strict_bit_exact(m):
    """ring2d-type case (128x128x3, IORD 2, zero-flux) for 64 steps."""
    import oracle
    r = workloads.ring2d(128)
    U, V, W = workloads.faces_from_cells(r["u"], r["v"], r["w"])
    U, V, W = (x.astype(np.float32) for x in (U, V, W))
    c = r["c0"].astype(np.float32)
    ref = c
    for _ in range(64):
        ref = oracle.step_faces(U, V, W, ref, 2)
    with m.Solver(128, 128, 3, order=2, strict=True) as s:
        s.set_faces(U, V, W)
        s.set_field(c)
        s.step(64)
        assert np.array_equal(s.get_field(), ref)
        mass = s.mass()
    assert abs(mass - oracle.mass(ref)) <= 1e-9 * abs(mass)


def test_ring3d_positivity_and_mass(m):
    """Limited ring3d-type flow: every cell stays >= 0 and the interior mass
    is conserved (zero-flux faces, no divergence) to FP32 accuracy."""
    r = workloads.ring3d(n=48, ns=48, courant=0.4, wcourant=0.0, sigma=4.0, offset=10.0)
    U, V, W = (x.astype(np.float32) for x in workloads.faces_from_cells(r["u"], r["v"], r["w"]))
    c = r["c0"].astype(np.float32)
    with m.Solver(48, 48, 48, order=2, limiter=True) as s:
        s.set_faces(U, V, W)
        s.set_field(c)
        m0 = s.mass()
        s.step(40)
        mn, nneg = s.min()
        m1 = s.mass()
    assert nneg == 0 and mn >= 0.0
    assert abs(m1 - m0) / m0 <= 1e-6


def test_fp32_form_against_fp64_plain_run(m):
    """ring3d-type case: FP32 storage with FP64 limiter ratios against an FP64
    run of the same scheme (relative L2 <= 1e-5)."""
    r = workloads.ring3d(n=40, ns=40, courant=0.4, wcourant=0.1, sigma=4.0, offset=8.0)
    U, V, W = workloads.faces_from_cells(r["u"], r["v"], r["w"])
    with m.Solver(40, 40, 40, order=2, dtype=np.float64, limiter=True) as s64:
        s64.set_faces(U, V, W)
        s64.set_field(r["c0"])
        s64.step(30)
        ref = s64.get_field()
    with m.Solver(40, 40, 40, order=2, limiter=True, precision_form=True) as s32:
        s32.set_faces(*(x.astype(np.float32) for x in (U, V, W)))
        s32.set_field(r["c0"].astype(np.float32))
        s32.step(30)
        got = s32.get_field().astype(np.float64)
        mn, nneg = s32.min()
    rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert rel <= 1e-5 and nneg == 0


def test_courant_check_rejects_unstable_faces(m):
    U = np.zeros((5, 6, 7), np.float32); V = np.zeros_like(U); W = np.zeros_like(U)
    U[2, 2, 3] = 1.5
    with m.Solver(7, 6, 5, order=2, check_courant=True) as s:
        with pytest.raises(m.MpdataError) as e:
            s.set_faces(U, V, W)
        assert e.value.code == -4
