import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA kernels")


def golden_files(floating_only=False):
    """Fixture paths; floating_only drops the INTEGER-build ones (int_*)."""
    files = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))
    if floating_only:
        files = [f for f in files if not os.path.basename(f).startswith("int_")]
    return files


def load_golden(path):
    z = np.load(path)
    return {k: (z[k] if z[k].shape != () else z[k].item()) for k in z.files}


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build(reference=True)
    return oracle


def integer_cases(oracle, shape, order, steps=1, count=3, limit=2 ** 31, **kw):
    """Seeded INTEGER-build cases (workloads.integer_case) the oracle runs for
    `steps` driver-style steps without a division by zero (where the
    reference traps) and with every value below `limit` (far from 64-bit
    overflow, where its behaviour is undefined).  Returns (seed, case,
    [(newest, other) per step]) tuples."""
    from mpdata_b200 import workloads
    nx, ny, ns = shape
    kw.setdefault("cmax", 1000)
    kw.setdefault("moving", 0.02)
    out = []
    for seed in range(4000):
        g = workloads.integer_case(nx, ny, ns, seed=seed, **kw)
        c0, c1 = g["c0"].copy(), np.zeros_like(g["c0"])
        res = []
        for _ in range(steps):
            rc, newest, other = oracle.smolar(g["dx"], g["dy"], g["ds"], g["dt"], g["u0"],
                                              g["u1"], g["v0"], g["v1"], g["w0"], g["w1"], c0,
                                              c1, order, dtype=np.int64)
            if rc != 0 or max(np.abs(newest).max(), np.abs(other).max()) >= limit:
                res = None
                break
            res.append((newest.copy(), other.copy()))
            c0, c1 = newest.copy(), other.copy()
        if res:
            out.append((seed, g, res))
            if len(out) == count:
                break
    return out
