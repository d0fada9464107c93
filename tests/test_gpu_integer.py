"""smolar_i64(): the reference's INTEGER build (real = long, ONE 4, HALF 2,
QUAT 1, MINVAL 1) on the GPU.

Integer arithmetic leaves no rounding to argue about: the GPU results must
equal the reference's bit for bit -- on the golden fixtures made by the
reference's own INTEGER build (tests/golden/int_*.npz) and on fresh seeded
cases checked against the oracle, over several driver-style steps (the newest
output becomes the next input), with the reference's pointer exchange.
Cases are those the oracle runs without a division by zero (where the
reference traps) and far from 64-bit overflow; a case that does divide by
zero must fail with MPDATA_ERR_INT_DIV0 and leave the caller's arrays alone.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, integer_cases, load_golden
from mpdata_b200 import workloads

pytestmark = pytest.mark.gpu

INT_GOLDEN = sorted(f for f in os.listdir(GOLDEN) if f.startswith("int_"))


@pytest.fixture(scope="module")
def m():
    import mpdata_b200
    return mpdata_b200


def _steps(m, g, order, steps):
    nx = g["c0"].shape[2]; ny = g["c0"].shape[1]; ns = g["c0"].shape[0]
    c0, c1 = g["c0"].copy(), np.zeros_like(g["c0"])
    out = []
    for _ in range(steps):
        a, b = m.smolar(nx, ny, ns, g["dx"], g["dy"], g["ds"], g["dt"], g["u0"], g["u1"],
                        g["v0"], g["v1"], g["w0"], g["w1"], c0, c1, order=order,
                        dtype=np.int64)
        out.append((b.copy(), a.copy(), b is c1))  # newest, other, newest in c1's array
        c0, c1 = b, a
    return out


def test_integer_golden_fixtures_exist():
    assert len(INT_GOLDEN) >= 5


@pytest.mark.parametrize("name", INT_GOLDEN)
def test_smolar_i64_matches_reference_golden(m, name):
    g = load_golden(os.path.join(GOLDEN, name))
    got = _steps(m, g, int(g["order"]), int(g["steps"]))
    newest, other, in_c1 = got[-1]
    assert np.array_equal(newest, g["newest"])
    assert np.array_equal(other, g["other"])


@pytest.mark.parametrize("shape,order,steps", [((17, 13, 11), 1, 3), ((9, 7, 5), 2, 2),
                                               ((9, 7, 5), 3, 1), ((9, 7, 5), 4, 1),
                                               ((12, 10, 8), 2, 2), ((33, 3, 6), 2, 1),
                                               ((3, 3, 3), 3, 1), ((40, 9, 4), 1, 2)])
def test_smolar_i64_matches_oracle(m, oracle_mod, shape, order, steps):
    cases = integer_cases(oracle_mod, shape, order, steps=steps, count=3)
    assert cases
    for seed, g, expect in cases:
        got = _steps(m, g, order, steps)
        for (newest, other, in_c1), (en, eo) in zip(got, expect):
            assert np.array_equal(newest, en), seed
            assert np.array_equal(other, eo), seed
            assert in_c1 == bool(order & 1)  # pointers exchanged iff order is even


def test_smolar_i64_reports_division_by_zero(m, oracle_mod):
    """A case the reference would trap on: MPDATA_ERR_INT_DIV0, arrays untouched."""
    for seed in range(200):
        g = workloads.integer_case(9, 7, 5, seed=seed)
        c0, c1 = g["c0"].copy(), np.zeros_like(g["c0"])
        rc, _, _ = oracle_mod.smolar(g["dx"], g["dy"], g["ds"], g["dt"], g["u0"], g["u1"],
                                     g["v0"], g["v1"], g["w0"], g["w1"], c0, c1, 3,
                                     dtype=np.int64)
        if rc == -2:
            break
    else:
        pytest.fail("no zero-divisor case found")
    c0 = g["c0"].copy()
    c1 = np.full_like(c0, 123)
    with pytest.raises(m.MpdataError) as e:
        m.smolar(9, 7, 5, g["dx"], g["dy"], g["ds"], g["dt"], g["u0"], g["u1"], g["v0"], g["v1"],
                 g["w0"], g["w1"], c0, c1, order=3, dtype=np.int64)
    assert e.value.code == -6
    assert np.array_equal(c0, g["c0"]) and (c1 == 123).all()
    # the next call starts clean
    good = integer_cases(oracle_mod, (9, 7, 5), 2, steps=1, count=1)[0]
    got = _steps(m, good[1], 2, 1)
    assert np.array_equal(got[0][0], good[2][0][0])


def test_smolar_i64_zero_grid_step_is_division_by_zero(m):
    """dx = 0: QUAT dt / dx divides by zero in the reference's uu_init (uu.c:132)."""
    g = workloads.integer_case(6, 5, 4, seed=3)
    g["dx"][2] = 0
    with pytest.raises(m.MpdataError) as e:
        _steps(m, g, 1, 1)
    assert e.value.code == -6
