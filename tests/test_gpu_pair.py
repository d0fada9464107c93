"""The two-cells-per-thread corrective pass (FP32, default arithmetic).

It regroups the reference's face formulas (shared face sums, per-cell
divergence terms, exchanged fluxes), so it is compared with the oracle within
the default-mode FP32 tolerance rather than bit for bit:

  max |gpu - oracle| <= 1e-5 after 2 steps (fields O(1))
  z-chunked marches: bit-identical to the unchunked march
  with the limiter: no negative values, mass kept to 1e-6 (zero-flux case)

Grids are chosen so the CTA grid has both interior CTAs (the branch-free
path) and boundary CTAs, with partial CTAs at the high ends.
"""
import numpy as np
import pytest

from mpdata_b200 import workloads

pytestmark = pytest.mark.gpu

TOL = 1e-5
SHAPES = [(130, 100, 12), (67, 45, 9), (200, 37, 3), (35, 34, 5), (3, 3, 3), (96, 70, 40)]
OPTS = [dict(), dict(limiter=1), dict(vv_fix=1), dict(div_mode=1), dict(limiter=1, vv_fix=1)]


@pytest.fixture(scope="module")
def m():
    import mpdata_b200
    yield mpdata_b200


def _faces(case):
    import oracle
    U, V, W = oracle.courant(case["dx"], case["dy"], case["ds"], case["dt"], case["u0"],
                             case["u1"], case["v0"], case["v1"], case["w0"], case["w1"],
                             dtype=np.float64)
    return U.astype(np.float32), V.astype(np.float32), W.astype(np.float32)


def _run(m, shape, order, opt, steps, approx=False, kernel=3, depth=None, seed=0,
         precision_form=False):
    nx, ny, ns = shape
    case = workloads.random_case(nx, ny, ns, seed=seed)
    U, V, W = _faces(case)
    c = case["c0"].astype(np.float32)
    with m.Solver(nx, ny, ns, order=order, limiter=bool(opt.get("limiter")),
                  vv_fix=bool(opt.get("vv_fix")), div_mode=opt.get("div_mode", 0),
                  approx_div=approx, kernel=kernel, precision_form=precision_form) as s:
        if depth is not None:
            s.set_march_depth(depth)
        s.set_faces(U, V, W)
        s.set_field(c)
        s.step(steps)
        return s.get_field(), (U, V, W, c)


@pytest.mark.parametrize("approx", [False, True], ids=["ieee", "approx"])
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("order", [1, 2, 3, 4])
@pytest.mark.parametrize("opt", OPTS, ids=lambda o: "-".join(o) or "plain")
def test_pair_pass_within_tolerance(m, approx, shape, order, opt):
    import oracle
    got, (U, V, W, c) = _run(m, shape, order, opt, 2, approx=approx, seed=sum(shape) + order)
    ref = c
    for _ in range(2):
        ref = oracle.step_faces(U, V, W, ref, order, **opt)
    err = float(np.abs(got - ref).max())
    assert err <= TOL, err


@pytest.mark.parametrize("shape", [(130, 100, 12), (67, 45, 9)], ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("opt", OPTS[:2], ids=lambda o: "-".join(o) or "plain")
def test_pair_pass_agrees_with_one_cell_pass(m, shape, opt):
    a, _ = _run(m, shape, 3, opt, 3, kernel=3, seed=5)
    b, _ = _run(m, shape, 3, opt, 3, kernel=2, seed=5)
    assert float(np.abs(a - b).max()) <= TOL


FORMS = {"ieee": dict(), "approx": dict(approx=True),
         "precision": dict(approx=True, precision_form=True)}


@pytest.mark.parametrize("depth", [1, 2, 3, 7, 0])
@pytest.mark.parametrize("limiter", [0, 1])
@pytest.mark.parametrize("form", list(FORMS))
def test_pair_pass_z_chunks_bit_identical(m, depth, limiter, form):
    """A march split into z chunks of any depth equals the whole-column
    march bit for bit, for the unrolled (approx_div) and the rolled (IEEE,
    precision) plane loops."""
    if form == "precision" and not limiter:
        pytest.skip("the precision form acts on the limiter")
    shape = (70, 40, 26)
    full, _ = _run(m, shape, 3, dict(limiter=limiter), 2, depth=0, seed=9, **FORMS[form])
    got, _ = _run(m, shape, 3, dict(limiter=limiter), 2, depth=depth, seed=9, **FORMS[form])
    assert np.array_equal(full, got)


def test_pair_pass_limiter_positive_and_conservative(m):
    """ring3d-type flow with zero-flux boundaries, 96^2 x 40 (interior and
    boundary CTAs): every cell stays >= 0, mass kept to 1e-6."""
    r = workloads.ring3d(n=96, ns=40, courant=0.4, wcourant=0.0, sigma=6.0, offset=20.0)
    U, V, W = (x.astype(np.float32) for x in workloads.faces_from_cells(r["u"], r["v"], r["w"]))
    with m.Solver(96, 96, 40, order=3, limiter=True, approx_div=True) as s:
        s.set_faces(U, V, W)
        s.set_field(r["c0"].astype(np.float32))
        m0 = s.mass()
        s.step(40)
        mn, nneg = s.min()
        m1 = s.mass()
    assert nneg == 0 and mn >= 0.0
    assert abs(m1 - m0) / m0 <= 1e-6


@pytest.mark.parametrize("approx", [False, True], ids=["ieee", "approx"])
def test_pair_pass_against_fp64_run(m, approx):
    """Streamfunction flow and lognormal field (the throughput workload's
    kind, 160 x 140 x 24): FP32 two-cell pass against the FP64 solver,
    relative L2 <= 1e-5 after 10 steps of IORD 3 with the limiter."""
    w = workloads.roofline(160, 140, 24)
    with m.Solver(160, 140, 24, order=3, dtype=np.float64, limiter=True) as s64:
        s64.set_faces(w["U"], w["V"], w["W"])
        s64.set_field(w["c0"])
        s64.step(10)
        ref = s64.get_field()
    with m.Solver(160, 140, 24, order=3, limiter=True, approx_div=approx, kernel=3) as s32:
        s32.set_faces(*(w[k].astype(np.float32) for k in ("U", "V", "W")))
        s32.set_field(w["c0"].astype(np.float32))
        s32.step(10)
        got = s32.get_field().astype(np.float64)
        mn, nneg = s32.min()
    rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert rel <= 1e-5 and nneg == 0, rel


@pytest.mark.parametrize("approx", [False, True], ids=["ieee", "approx"])
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("order", [2, 3])
def test_pair_precision_form_within_tolerance(m, approx, shape, order):
    """The precision form on the two-cell pass (FP64 limiter sums and ratios)
    against the oracle's precision form (wide_beta)."""
    import oracle
    opt = dict(limiter=1)
    got, (U, V, W, c) = _run(m, shape, order, opt, 2, approx=approx, seed=sum(shape) + 3 * order,
                             precision_form=True)
    ref = c
    for _ in range(2):
        ref = oracle.step_faces(U, V, W, ref, order, limiter=1, wide_beta=1)
    err = float(np.abs(got - ref).max())
    assert err <= TOL, err


@pytest.mark.parametrize("depth", [1, 5, 0])
def test_pair_precision_form_z_chunks_bit_identical(m, depth):
    shape = (70, 40, 26)
    full, _ = _run(m, shape, 3, dict(limiter=1), 2, approx=True, depth=0, seed=9,
                   precision_form=True)
    got, _ = _run(m, shape, 3, dict(limiter=1), 2, approx=True, depth=depth, seed=9,
                  precision_form=True)
    assert np.array_equal(full, got)


@pytest.mark.parametrize("approx", [False, True], ids=["ieee", "approx"])
def test_pair_precision_form_near_zero_fields(m, approx):
    """A field spanning 1 down to subnormal values, with exact zeros, so that
    limiter sums fall below 2^-100 and take the precision form's FP64 path:
    the result stays finite, non-negative and within max-abs 1e-5 of the
    oracle's precision form."""
    import oracle
    nx, ny, ns = 70, 40, 12
    case = workloads.random_case(nx, ny, ns, seed=31)
    U, V, W = _faces(case)
    rng = np.random.default_rng(32)
    c = (rng.uniform(0.0, 1.0, (ns, ny, nx)) * 10.0 ** rng.integers(-44, 1, (ns, ny, nx)))
    c[rng.random(c.shape) < 0.2] = 0.0
    c = c.astype(np.float32)
    with m.Solver(nx, ny, ns, order=2, limiter=True, approx_div=approx, kernel=3,
                  precision_form=True) as s:
        s.set_faces(U, V, W)
        s.set_field(c)
        s.step(2)
        got = s.get_field()
    ref = c
    for _ in range(2):
        ref = oracle.step_faces(U, V, W, ref, 2, limiter=1, wide_beta=1)
    assert np.isfinite(got).all() and float(got.min()) >= 0.0
    assert float(np.abs(got - ref).max()) <= TOL


@pytest.mark.parametrize("seed", [1, 2])
def test_division_matches_ieee_bit_for_bit(m, seed):
    """The IEEE form of the two-cell pass divides without the compiled
    division's slow path (Newton-refined hardware reciprocal and Markstein's
    remainder correction, IEEE division only for near-zero numerators): on
    2^32 seeded operand pairs of the pass's ranges (divisors FLT_MIN..2^100,
    numerators of either sign from zero and subnormals up), plain and clamped
    to 1, every result equals IEEE round-to-nearest division bit for bit."""
    assert m.check_division(1 << 32, seed) == 0
