"""Host-side logic of the decomposed step (msmolar), checked on the CPU with
the oracle: the reference's block sizing rule, and the halo depth that makes
a blocked step bit-identical to the single-domain step (P cells without the
limiter, 2P-1 with it), while one cell less is not enough."""
import numpy as np
import pytest

from mpdata_b200 import workloads


def split_axis(n, s):
    """Block starts: n // s cells each, the first n % s blocks one more
    (reference multigrid/src/grid.c:68-144)."""
    s = min(s, n)
    base, rem = divmod(n, s)
    st = [0]
    for b in range(s):
        st.append(st[-1] + base + (1 if b < rem else 0))
    return st


def halo_depth(order, limiter):
    return order + (order - 1 if limiter else 0)


def blocked_step(oracle, U, V, W, c, order, split, halo, limiter):
    ns, ny, nx = c.shape
    starts = [split_axis(n, s) for n, s in zip((nx, ny, ns), split)]
    out = c.copy()
    for bz in range(len(starts[2]) - 1):
        for by in range(len(starts[1]) - 1):
            for bx in range(len(starts[0]) - 1):
                lo = [starts[a][b] for a, b in enumerate((bx, by, bz))]
                hi = [starts[a][b + 1] for a, b in enumerate((bx, by, bz))]
                n = (nx, ny, ns)
                elo = [max(0, l - halo) for l in lo]
                ehi = [min(n[a], hi[a] + halo) for a in range(3)]
                if min(ehi[a] - elo[a] for a in range(3)) < 3:
                    continue  # owns shell cells only: they never change
                sl = (slice(elo[2], ehi[2]), slice(elo[1], ehi[1]), slice(elo[0], ehi[0]))
                res = oracle.step_faces(*(np.ascontiguousarray(x[sl]) for x in (U, V, W)),
                                        np.ascontiguousarray(c[sl]), order, limiter=limiter)
                own = tuple(slice(lo[a] - elo[a], hi[a] - elo[a]) for a in (2, 1, 0))
                out[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] = res[own]
    return out


def test_split_axis_matches_reference_rule():
    assert split_axis(10, 3) == [0, 4, 7, 10]
    assert split_axis(7, 7) == list(range(8))
    assert split_axis(5, 9) == list(range(6))  # clamped like grid.c:34-36


@pytest.mark.parametrize("order,limiter", [(1, 0), (2, 0), (3, 0), (2, 1), (3, 1)])
def test_halo_depth_gives_exact_decomposition(oracle_mod, order, limiter):
    case = workloads.random_case(22, 19, 17, seed=order + 10 * limiter)
    U, V, W = oracle_mod.courant(case["dx"], case["dy"], case["ds"], case["dt"], case["u0"],
                                 case["u1"], case["v0"], case["v1"], case["w0"], case["w1"],
                                 dtype=np.float64)
    c = case["c0"]
    h = halo_depth(order, limiter)
    ref = c.copy()
    blk = c.copy()
    short = c.copy()
    for _ in range(3):
        ref = oracle_mod.step_faces(U, V, W, ref, order, limiter=limiter)
        blk = blocked_step(oracle_mod, U, V, W, blk, order, (3, 2, 2), h, limiter)
        short = blocked_step(oracle_mod, U, V, W, short, order, (3, 2, 2), h - 1, limiter)
    assert np.array_equal(blk, ref)
    if h > 1 or order > 1:
        assert not np.array_equal(short, ref)
