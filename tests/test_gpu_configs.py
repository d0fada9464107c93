"""GPU parity on the benchmark configurations at their own sizes and lengths.

* ring2d (128 x 128, reference form 128 x 128 x 3), IORD 2, no limiter,
  1024 steps through smolar(): strict arithmetic bit-identical to the
  reference's own smolar() built from its sources (oracle/_ref) at several
  points of the run and at its end, which crosses the steps where the field
  reaches the x = 1 column that vv_pass leaves unwritten (core/src/vv.c:81-82);
  default arithmetic within max-abs 1e-5.  The reference's unmodified ring2d
  driver at its own command line (`ring2d 128 1024`, tests/ring2d/test.c:45-64),
  linked against this library, writes the same bytes as when linked against
  the reference core.
* ring3d (128^3, 128 steps, IORD 2 + limiter, tests/ring3d/test.c:24 with the
  flow of the configuration): the FP64 GPU run in strict arithmetic equals
  the FP64 oracle bit for bit after 128 steps; the FP32 forms (plain, the
  precision form, approx_div) stay within relative L2 1e-5 of it with no
  negative cell; zero-flux mass drift <= 1e-6 (FP32) and 1e-12 (FP64).
  The same checks with the y faces of the x = 1 column computed (vv_fix)
  against the FP64 oracle under that rule.
* the throughput grid (512 x 512 x 256), plain IORD 3 without the limiter (the
  reference has none), 2 steps through smolar(): strict arithmetic
  bit-identical to the reference's own smolar(); default arithmetic within
  max-abs 1e-5 x max|c| (relative to the field's largest value) and relative
  L2 1e-6.
"""
import os
import subprocess

import numpy as np
import pytest

from mpdata_b200 import workloads

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = os.path.join(ROOT, "oracle", "_ref")


@pytest.fixture(scope="module")
def m():
    import mpdata_b200
    yield mpdata_b200
    mpdata_b200.set_default_options(None)


def _ref_or_skip(oracle_mod, variant):
    if not oracle_mod.ref_available(variant):
        pytest.skip(f"oracle/_ref/libref_{variant}.so not built (no reference checkout at build)")


def _run_smolar(step, c, steps, marks=()):
    """Driver loop of tests/ring2d/test.c:45-64: after each call the newest
    field becomes the next input.  Returns the newest field and copies at the
    steps in `marks`."""
    c0 = c.copy()
    c1 = np.zeros_like(c0)
    seen = {}
    for it in range(1, steps + 1):
        newest, other = step(c0, c1)
        c0, c1 = newest, other
        if it in marks:
            seen[it] = newest.copy()
    return c0, seen


def _ring2d_inputs():
    r = workloads.ring2d(128)
    f = {k: np.ascontiguousarray(r[k], np.float32) for k in ("u", "v", "w", "c0")}
    one = np.ones(128, np.float32), np.ones(128, np.float32), np.ones(3, np.float32)
    return f, one


MARKS = (200, 227, 256, 300, 512, 1024)


def test_ring2d_1024_steps_strict_equals_reference_build(m, oracle_mod):
    _ref_or_skip(oracle_mod, "f32")
    f, (dx, dy, ds) = _ring2d_inputs()
    vel = (f["u"], f["u"], f["v"], f["v"], f["w"], f["w"])
    col1 = []

    def ref_step(c0, c1):
        _, newest, other = oracle_mod.ref_smolar(dx, dy, ds, 1.0, *vel, c0, c1, 2, variant="f32")
        col1.append(float(np.abs(newest[1, 1:-1, 1]).max()))
        return newest, other

    def gpu_step(c0, c1):
        a, b = m.smolar(128, 128, 3, dx, dy, ds, 1.0, *vel, c0, c1, order=2)
        return b, a

    ref, ref_marks = _run_smolar(ref_step, f["c0"], 1024, MARKS)
    # the rotating blob brings values of order 1e-3 to the column vv_pass
    # leaves unwritten (x = 1) during the run
    assert max(col1) > 1e-3
    m.set_default_options(m.SolverOptions(strict=True))
    try:
        got, got_marks = _run_smolar(gpu_step, f["c0"], 1024, MARKS)
    finally:
        m.set_default_options(None)
    for it in MARKS:
        assert np.array_equal(got_marks[it], ref_marks[it]), it
    assert np.array_equal(got, ref)
    # default arithmetic (FMA contraction): within FP32 rounding after 1024 steps
    dflt, _ = _run_smolar(gpu_step, f["c0"], 1024)
    assert float(np.abs(dflt - ref).max()) <= 1e-5


def test_reference_ring2d_driver_full_length(tmp_path):
    """`ring2d 128 1024`: the reference's own CPU case, unmodified driver."""
    exe_ref = os.path.join(REF_BIN, "ring2d_ref")
    exe_gpu = os.path.join(REF_BIN, "ring2d_b200")
    if not (os.path.exists(exe_ref) and os.path.exists(exe_gpu)):
        pytest.skip("reference ring2d drivers not built")
    ref, gpu = tmp_path / "ref", tmp_path / "gpu"
    ref.mkdir(), gpu.mkdir()
    env = dict(os.environ)
    env.pop("MPDATA_B200_OPTIONS", None)
    p1 = subprocess.run([exe_ref, "128", "1024"], cwd=ref, env=env, capture_output=True,
                        text=True, timeout=600)
    env["MPDATA_B200_OPTIONS"] = "strict"
    p2 = subprocess.run([exe_gpu, "128", "1024"], cwd=gpu, env=env, capture_output=True,
                        text=True, timeout=600)
    assert p1.returncode == 0 and p2.returncode == 0, (p1.stderr, p2.stderr)
    assert p1.stdout == p2.stdout
    assert (ref / "ring2d.bin").read_bytes() == (gpu / "ring2d.bin").read_bytes()


# ---- ring3d: 128^3, 128 steps, IORD 2 + limiter --------------------------

N3, STEPS3 = 128, 128


@pytest.fixture(scope="module")
def ring3d_case():
    r = workloads.ring3d(n=N3)
    U, V, W = workloads.faces_from_cells(r["u"], r["v"], r["w"])
    # both precisions step from the same (FP32-representable) inputs
    U, V, W, c0 = (np.ascontiguousarray(x.astype(np.float32), np.float64)
                   for x in (U, V, W, r["c0"]))
    return U, V, W, c0


@pytest.fixture(scope="module")
def ring3d_fp64(ring3d_case, oracle_mod):
    U, V, W, c = ring3d_case
    for _ in range(STEPS3):
        c = oracle_mod.step_faces(U, V, W, c, 2, limiter=1)
    return c


def _solver_run(m, case, dtype, steps, **opts):
    U, V, W, c0 = case
    with m.Solver(N3, N3, N3, order=2, dtype=dtype, limiter=True, **opts) as s:
        s.set_faces(*(np.ascontiguousarray(x, dtype) for x in (U, V, W)))
        s.set_field(np.ascontiguousarray(c0, dtype))
        m0 = s.mass()
        s.step(steps)
        mn, nneg = s.min()
        return s.get_field().astype(np.float64), m0, s.mass(), mn, nneg


def test_ring3d_fp64_strict_equals_oracle(m, ring3d_case, ring3d_fp64):
    got, m0, m1, mn, nneg = _solver_run(m, ring3d_case, np.float64, STEPS3, strict=True)
    assert np.array_equal(got, ring3d_fp64)
    assert nneg == 0 and mn >= 0.0
    assert abs(m1 - m0) / m0 <= 1e-12


@pytest.mark.parametrize("form", [dict(), dict(precision_form=True, approx_div=True),
                                  dict(approx_div=True)],
                         ids=["plain", "precision_form", "approx_div"])
def test_ring3d_fp32_forms_against_fp64(m, ring3d_case, ring3d_fp64, form):
    got, m0, m1, mn, nneg = _solver_run(m, ring3d_case, np.float32, STEPS3, **form)
    rel = float(np.linalg.norm(got - ring3d_fp64) / np.linalg.norm(ring3d_fp64))
    assert rel <= 1e-5, rel
    assert nneg == 0 and mn >= 0.0
    assert abs(m1 - m0) / m0 <= 1e-6, abs(m1 - m0) / m0


# The same configuration with the y faces of the x = 1 column computed
# (vv_fix) instead of the reference's buffer rule for the column vv_pass
# leaves unwritten: the FP64 oracle and the GPU under that rule.

@pytest.fixture(scope="module")
def ring3d_fp64_fix(ring3d_case, oracle_mod):
    U, V, W, c = ring3d_case
    for _ in range(STEPS3):
        c = oracle_mod.step_faces(U, V, W, c, 2, limiter=1, vv_fix=1)
    return c


def test_ring3d_column_rule_fp64_strict_equals_oracle(m, ring3d_case, ring3d_fp64_fix):
    got, m0, m1, mn, nneg = _solver_run(m, ring3d_case, np.float64, STEPS3, strict=True,
                                        vv_fix=True)
    assert np.array_equal(got, ring3d_fp64_fix)
    assert nneg == 0 and mn >= 0.0
    assert abs(m1 - m0) / m0 <= 1e-12


@pytest.mark.parametrize("form", [dict(), dict(precision_form=True, approx_div=True),
                                  dict(approx_div=True)],
                         ids=["plain", "precision_form", "approx_div"])
def test_ring3d_column_rule_fp32_forms_against_fp64(m, ring3d_case, ring3d_fp64_fix, form):
    got, m0, m1, mn, nneg = _solver_run(m, ring3d_case, np.float32, STEPS3, vv_fix=True, **form)
    rel = float(np.linalg.norm(got - ring3d_fp64_fix) / np.linalg.norm(ring3d_fp64_fix))
    assert rel <= 1e-5, rel
    assert nneg == 0 and mn >= 0.0
    assert abs(m1 - m0) / m0 <= 1e-6, abs(m1 - m0) / m0


# ---- the throughput grid against the reference build ----------------------

@pytest.fixture(scope="module")
def fullsize_cells():
    wl = workloads.roofline(512, 512, 256)
    u, v, w = (np.ascontiguousarray(x, np.float32)
               for x in workloads.cell_velocities(wl["U"], wl["V"], wl["W"]))
    return u, v, w, np.ascontiguousarray(wl["c0"], np.float32)


def test_fullsize_plain_two_steps_against_reference_build(m, oracle_mod, fullsize_cells):
    _ref_or_skip(oracle_mod, "f32")
    u, v, w, c = fullsize_cells
    nx, ny, ns = 512, 512, 256
    dx, dy, ds = np.ones(nx, np.float32), np.ones(ny, np.float32), np.ones(ns, np.float32)
    vel = (u, u, v, v, w, w)

    def ref_step(c0, c1):
        _, newest, other = oracle_mod.ref_smolar(dx, dy, ds, 1.0, *vel, c0, c1, 3, variant="f32")
        return newest, other

    def gpu_step(c0, c1):
        a, b = m.smolar(nx, ny, ns, dx, dy, ds, 1.0, *vel, c0, c1, order=3)
        return b, a

    ref, _ = _run_smolar(ref_step, c, 2)
    m.set_default_options(m.SolverOptions(strict=True))
    try:
        got, _ = _run_smolar(gpu_step, c, 2)
    finally:
        m.set_default_options(None)
    assert np.array_equal(got, ref)
    dflt, _ = _run_smolar(gpu_step, c, 2)
    scale = float(np.abs(ref).max())
    assert float(np.abs(dflt - ref).max()) <= 1e-5 * scale
    rel = np.linalg.norm(dflt.astype(np.float64) - ref) / np.linalg.norm(ref.astype(np.float64))
    assert rel <= 1e-6, rel
