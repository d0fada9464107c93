"""GPU tests of the batched 2D ensemble (mpdata_ensemble_*).

Each instance is checked against the single-grid solver on the reference's
3-plane 2D form (nx x ny x 3, w = 0): in strict arithmetic the values are
identical (np.array_equal), for every tile-shape candidate, with the graph
replay and with direct launches; the default arithmetic stays within the
float32 tolerance (max abs <= 1e-5).
"""
import numpy as np
import pytest

from mpdata_b200 import workloads

pytestmark = pytest.mark.gpu

SIZES = [(5, 7), (70, 40), (33, 9), (129, 66), (3, 3), (64, 200)]


def _instances(seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for nx, ny in SIZES:
        U = np.zeros((ny, nx)); V = np.zeros((ny, nx))
        U[1:-1, :-1] = rng.uniform(-0.3, 0.3, (ny - 2, nx - 1))
        V[:-1, 1:-1] = rng.uniform(-0.3, 0.3, (ny - 1, nx - 2))
        c = rng.uniform(0.0, 1.0, (ny, nx))
        out.append(dict(nx=nx, ny=ny, U=U.astype(np.float32), V=V.astype(np.float32),
                        c0=c.astype(np.float32)))
    return out


def _three_plane(m, inst, steps, order, **opts):
    nx, ny = inst["nx"], inst["ny"]
    U = np.zeros((3, ny, nx), np.float32); V = np.zeros_like(U); W = np.zeros_like(U)
    U[1] = inst["U"]; V[1] = inst["V"]
    c = np.repeat(inst["c0"][None], 3, 0)
    with m.Solver(nx, ny, 3, order=order, **opts) as s:
        s.set_faces(U, V, W)
        s.set_field(c)
        s.step(steps)
        return s.get_field()[1]


@pytest.mark.parametrize("tile", [0, 1, 2, 3])
@pytest.mark.parametrize("limiter", [0, 1])
@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("graph", [True, False], ids=["graph", "direct"])
def test_ensemble_strict_equals_three_plane_solver(tile, limiter, order, graph):
    import mpdata_b200 as m
    insts = _instances(seed=order + 3 * limiter)
    opts = dict(strict=True, limiter=bool(limiter))
    with m.Ensemble([d["nx"] for d in insts], [d["ny"] for d in insts], order=order, **opts) as e:
        e.set_tile(tile)
        for q, d in enumerate(insts):
            e.set_faces(q, d["U"], d["V"])
            e.set_field(q, d["c0"])
        e.step(2, graph=graph)
        e.step(1, graph=graph)
        got = [e.get_field(q) for q in range(len(insts))]
    for q, d in enumerate(insts):
        ref = _three_plane(m, d, 3, order, **opts)
        assert np.array_equal(got[q], ref), (q, np.abs(got[q] - ref).max())


@pytest.mark.parametrize("approx", [False, True])
def test_ensemble_default_within_tolerance(approx):
    import mpdata_b200 as m
    insts = _instances(seed=9)
    with m.Ensemble([d["nx"] for d in insts], [d["ny"] for d in insts], order=2, limiter=True,
                    approx_div=approx) as e:
        for q, d in enumerate(insts):
            e.set_faces(q, d["U"], d["V"])
            e.set_field(q, d["c0"])
        e.step(4)
        got = [e.get_field(q) for q in range(len(insts))]
    for q, d in enumerate(insts):
        ref = _three_plane(m, d, 4, 2, strict=True, limiter=True)
        assert np.abs(got[q] - ref).max() <= 1e-5


def test_ensemble_autotune_picks_a_candidate_and_keeps_results():
    import mpdata_b200 as m
    cfg = workloads.ensemble(n=12, lo=64, hi=160, seed=5)
    nx = [d["nx"] for d in cfg]; ny = [d["ny"] for d in cfg]
    with m.Ensemble(nx, ny, order=2, limiter=True, strict=True) as e:
        for q, d in enumerate(cfg):
            e.set_faces(q, d["U"].astype(np.float32), d["V"].astype(np.float32))
            e.set_field(q, d["c0"].astype(np.float32))
        tile, ms = e.autotune(trial_steps=3)
        assert tile in (0, 1, 2, 3) and ms > 0
        for q, d in enumerate(cfg):  # the trials advanced the fields: set them again
            e.set_field(q, d["c0"].astype(np.float32))
        e.step(5)
        got = e.get_field(3)
    d = cfg[3]
    ref = _three_plane(m, dict(nx=d["nx"], ny=d["ny"], U=d["U"].astype(np.float32),
                               V=d["V"].astype(np.float32), c0=d["c0"].astype(np.float32)),
                       5, 2, strict=True, limiter=True)
    assert np.array_equal(got, ref)
    assert got.min() >= 0.0


@pytest.mark.parametrize("vv_fix", [False, True], ids=["ref_column", "vv_fix"])
@pytest.mark.parametrize("tile", [1, 3], ids=["tile", "march"])
@pytest.mark.parametrize("strict", [True, False], ids=["strict", "default"])
def test_ensemble_matches_cpu_oracle_sample(strict, tile, vv_fix):
    """A sample of the benchmark-kind instances (rotation, Gaussian blob,
    IORD 2 + limiter) against the CPU oracle on the 3-plane form directly:
    strict arithmetic bit-identical, default within max-abs 1e-5; under both
    rules for the y faces of the x = 1 column."""
    import oracle

    import mpdata_b200 as m
    cfg = workloads.ensemble(n=24, lo=64, hi=200, seed=17)
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    steps = 6
    with m.Ensemble([d["nx"] for d in cfg], [d["ny"] for d in cfg], order=2, limiter=True,
                    strict=strict, vv_fix=vv_fix) as e:
        e.set_tile(tile)
        for q, d in enumerate(cfg):
            e.set_faces(q, f32(d["U"]), f32(d["V"]))
            e.set_field(q, f32(d["c0"]))
        e.step(steps)
        got = {q: e.get_field(q) for q in (0, 5, 11, 23)}
    for q, g in got.items():
        d = cfg[q]
        U = np.zeros((3, d["ny"], d["nx"]), np.float32); V = np.zeros_like(U)
        U[1] = f32(d["U"]); V[1] = f32(d["V"])
        c = np.repeat(f32(d["c0"])[None], 3, 0)
        for _ in range(steps):
            c = oracle.step_faces(U, V, np.zeros_like(U), c, 2, limiter=1, vv_fix=int(vv_fix))
        if strict:
            assert np.array_equal(g, c[1]), q
        else:
            assert float(np.abs(g - c[1]).max()) <= 1e-5, q
