"""The CPU oracle is pinned before it is trusted.

* against the golden fixtures, produced by the reference's own smolar()
  compiled from its sources (tests/golden/make_golden.py): bit for bit;
* against the reference library itself on fresh random cases when the
  reference build (oracle/_ref) is present: bit for bit;
* the limiter extension (no reference counterpart) by its defining
  properties.
"""
import os

import numpy as np
import pytest

from conftest import golden_files, load_golden
from mpdata_b200 import workloads


def _run_oracle(oracle, g, dtype):
    c0 = g["c0"].astype(dtype).copy()
    c1 = np.zeros_like(c0)
    for _ in range(int(g["steps"])):
        rc, newest, other = oracle.smolar(g["dx"], g["dy"], g["ds"], float(g["dt"]), g["u0"],
                                          g["u1"], g["v0"], g["v1"], g["w0"], g["w1"], c0, c1,
                                          int(g["order"]), dtype=dtype)
        assert rc == 0
        c0, c1 = newest.copy(), other.copy()
    return c0, c1


@pytest.mark.parametrize("path", golden_files(), ids=os.path.basename)
def test_oracle_reproduces_golden(oracle_mod, path):
    g = load_golden(path)
    dtype = g["c0"].dtype
    newest, other = _run_oracle(oracle_mod, g, dtype)
    assert np.array_equal(newest, g["newest"])
    assert np.array_equal(other, g["other"])


def test_golden_covers_reference_quirk_column(oracle_mod):
    """The fixtures exercise the y-face column the reference leaves unwritten:
    switching to the computed column changes their results."""
    g = load_golden(os.path.join(os.path.dirname(golden_files()[0]),
                                 "rand_12x10x8_o3_s3_f64.npz"))
    c0 = g["c0"].copy()
    rc, newest, _ = oracle_mod.smolar(g["dx"], g["dy"], g["ds"], float(g["dt"]), g["u0"],
                                      g["u1"], g["v0"], g["v1"], g["w0"], g["w1"], c0,
                                      np.zeros_like(c0), 3, dtype=np.float64, vv_fix=1)
    assert rc == 0
    c_ref = g["c0"].copy()
    rc, newest_ref, _ = oracle_mod.smolar(g["dx"], g["dy"], g["ds"], float(g["dt"]), g["u0"],
                                          g["u1"], g["v0"], g["v1"], g["w0"], g["w1"], c_ref,
                                          np.zeros_like(c_ref), 3, dtype=np.float64)
    assert not np.array_equal(newest, newest_ref)


@pytest.mark.parametrize("variant", ["f32", "f64"])
@pytest.mark.parametrize("shape", [(17, 13, 11), (5, 4, 3), (33, 3, 6), (3, 3, 3)])
@pytest.mark.parametrize("order", [1, 2, 3, 5])
def test_oracle_matches_reference_build(oracle_mod, variant, shape, order):
    if not oracle_mod.ref_available(variant):
        pytest.skip("reference build (oracle/_ref) not present")
    dtype = np.float64 if variant == "f64" else np.float32
    nx, ny, ns = shape
    case = workloads.random_case(nx, ny, ns, seed=nx * 7 + order)
    cv = {k: (v.astype(dtype) if isinstance(v, np.ndarray) else v) for k, v in case.items()}
    a0 = cv["c0"].copy(); a1 = np.zeros_like(a0)
    b0 = cv["c0"].copy(); b1 = np.zeros_like(b0)
    args = (cv["dx"], cv["dy"], cv["ds"], cv["dt"], cv["u0"], cv["u1"], cv["v0"], cv["v1"],
            cv["w0"], cv["w1"])
    r_ref = oracle_mod.ref_smolar(*args, a0, a1, order, variant=variant)
    r_own = oracle_mod.smolar(*args, b0, b1, order, dtype=dtype)
    assert r_ref[0] == 0 and r_own[0] == 0
    assert (r_ref[1] is a1) == (r_own[1] is b1)  # same pointer exchange
    assert np.array_equal(r_ref[1], r_own[1])
    assert np.array_equal(r_ref[2], r_own[2])


def test_order_zero_exchanges_pointers(oracle_mod):
    case = workloads.random_case(6, 5, 4, seed=3)
    cv = {k: (v.astype(np.float32) if isinstance(v, np.ndarray) else v) for k, v in case.items()}
    c0 = cv["c0"].copy(); c1 = np.zeros_like(c0)
    rc, newest, other = oracle_mod.smolar(cv["dx"], cv["dy"], cv["ds"], cv["dt"], cv["u0"],
                                          cv["u1"], cv["v0"], cv["v1"], cv["w0"], cv["w1"], c0,
                                          c1, 0)
    assert rc == 0 and newest is c0 and other is c1


# ---- the reference's INTEGER build (real = long) ----

@pytest.mark.parametrize("shape,order,steps", [((17, 13, 11), 1, 3), ((9, 7, 5), 2, 2),
                                               ((9, 7, 5), 3, 1), ((9, 7, 5), 4, 1),
                                               ((33, 3, 6), 2, 1), ((3, 3, 3), 3, 1)])
def test_integer_oracle_matches_reference_build(oracle_mod, shape, order, steps):
    """Bit for bit against the reference compiled with -DINTEGER, on cases the
    oracle first runs without a division by zero (the reference traps there)."""
    if not oracle_mod.ref_available("i64"):
        pytest.skip("reference INTEGER build (oracle/_ref) not present")
    from conftest import integer_cases
    cases = integer_cases(oracle_mod, shape, order, steps=steps, count=3)
    assert cases, "no usable integer case"
    for _, g, expect in cases:
        args = (g["dx"], g["dy"], g["ds"], g["dt"], g["u0"], g["u1"], g["v0"], g["v1"],
                g["w0"], g["w1"])
        c0, c1 = g["c0"].copy(), np.zeros_like(g["c0"])
        for newest_o, other_o in expect:
            rc, newest, other = oracle_mod.ref_smolar(*args, c0, c1, order, variant="i64")
            assert rc == 0
            assert (newest is c1) == bool(order & 1)  # pointer exchange iff order even
            assert np.array_equal(newest, newest_o) and np.array_equal(other, other_o)
            c0, c1 = newest.copy(), other.copy()


def test_integer_oracle_flags_division_by_zero(oracle_mod):
    """The integer scheme is not positivity-preserving: some cases reach
    c_hi + c_lo + MINVAL = 0, where the reference's division traps; the
    oracle reports them (-2) instead of dividing."""
    rcs = set()
    for seed in range(40):
        g = workloads.integer_case(9, 7, 5, seed=seed)
        c0, c1 = g["c0"].copy(), np.zeros_like(g["c0"])
        rc, _, _ = oracle_mod.smolar(g["dx"], g["dy"], g["ds"], g["dt"], g["u0"], g["u1"],
                                     g["v0"], g["v1"], g["w0"], g["w1"], c0, c1, 3,
                                     dtype=np.int64)
        rcs.add(rc)
    assert rcs == {0, -2}


def test_integer_oracle_rejects_limiter(oracle_mod):
    g = workloads.integer_case(5, 4, 3, seed=1)
    c0, c1 = g["c0"].copy(), np.zeros_like(g["c0"])
    rc, _, _ = oracle_mod.smolar(g["dx"], g["dy"], g["ds"], g["dt"], g["u0"], g["u1"], g["v0"],
                                 g["v1"], g["w0"], g["w1"], c0, c1, 2, dtype=np.int64,
                                 limiter=1)
    assert rc == -1


def _ring_faces(n=24, ns=10, courant=0.4):
    r = workloads.ring3d(n=n, ns=ns, courant=courant, wcourant=0.1, sigma=3.0, offset=5.0,
                         background=1e-6)
    U, V, W = workloads.faces_from_cells(r["u"], r["v"], r["w"])
    return U, V, W, r["c0"]


@pytest.mark.parametrize("order", [2, 3])
def test_limiter_positivity_and_bounds(oracle_mod, order):
    U, V, W, c = _ring_faces()
    c_lidded = c.copy()
    for _ in range(20):
        c_lidded = oracle_mod.step_faces(U, V, W, c_lidded, order, limiter=1)
    # uniform w against closed lids compresses mass (new maxima are physical),
    # but the field stays non-negative
    assert c_lidded[1:-1, 1:-1, 1:-1].min() >= 0.0
    # divergence-free rotation: no new extrema either
    W[:] = 0.0
    cmax = c.max()
    for _ in range(20):
        c = oracle_mod.step_faces(U, V, W, c, order, limiter=1)
    inner = c[1:-1, 1:-1, 1:-1]
    assert inner.min() >= 0.0
    assert inner.max() <= cmax * (1 + 1e-12)


def test_limiter_conserves_mass_with_zero_flux(oracle_mod):
    U, V, W, c = _ring_faces()
    W[:] = 0.0  # pure rotation with closed boundaries
    m0 = oracle_mod.mass(c)
    for _ in range(10):
        c = oracle_mod.step_faces(U, V, W, c, 3, limiter=1)
    assert abs(oracle_mod.mass(c) - m0) / m0 < 1e-12


def test_limiter_removes_plain_undershoot(oracle_mod):
    """A sharp step advected by uniform flow: plain MPDATA overshoots, the
    limited scheme stays within the initial bounds."""
    ns, ny, nx = 3, 6, 40
    c = np.zeros((ns, ny, nx)); c[:, :, 5:15] = 1.0
    U = np.zeros_like(c); V = np.zeros_like(c); W = np.zeros_like(c)
    U[1:-1, 1:-1, :-1] = 0.35
    plain = c.copy(); lim = c.copy()
    for _ in range(30):
        plain = oracle_mod.step_faces(U, V, W, plain, 3)
        lim = oracle_mod.step_faces(U, V, W, lim, 3, limiter=1)
    assert plain[1, 1:-1, 1:-1].max() > 1.0 + 1e-6  # plain scheme is oscillatory here
    assert lim[1, 1:-1, 1:-1].max() <= 1.0 + 1e-12
    assert lim[1, 1:-1, 1:-1].min() >= 0.0


def test_wide_beta_close_to_plain_limiter(oracle_mod):
    U, V, W, c = _ring_faces()
    c32 = c.astype(np.float32)
    a = b = c32
    for _ in range(5):
        a = oracle_mod.step_faces(U.astype(np.float32), V.astype(np.float32),
                                  W.astype(np.float32), a, 2, limiter=1)
        b = oracle_mod.step_faces(U.astype(np.float32), V.astype(np.float32),
                                  W.astype(np.float32), b, 2, limiter=1, wide_beta=1)
    assert np.abs(a - b).max() < 1e-5
