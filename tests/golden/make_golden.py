"""Generate the golden fixtures of this directory from the reference itself.

Runs the reference's own smolar() and test_init(), compiled unmodified from
the reference sources by oracle/Makefile (strict IEEE flags, vv.c with the
zero-filled allocation shim), on small seeded cases and stores inputs and
outputs as .npz files.  Needs the reference checkout (make -C oracle ref);
the fixtures themselves are committed so the tests run without it.

    python tests/golden/make_golden.py            # floating-point fixtures
    python tests/golden/make_golden.py integer    # INTEGER-build fixtures
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from mpdata_b200.workloads import integer_case, random_case  # noqa: E402

DTYPES = {"f32": np.float32, "f64": np.float64, "i64": np.int64}


def run_ref(case, order, variant, steps=1):
    dtype = DTYPES[variant]
    cv = {k: (np.ascontiguousarray(v, dtype) if isinstance(v, np.ndarray) else v)
          for k, v in case.items()}
    c0 = cv["c0"].copy()
    c1 = np.zeros_like(c0)
    for _ in range(steps):
        rc, newest, other = oracle.ref_smolar(cv["dx"], cv["dy"], cv["ds"], cv["dt"], cv["u0"],
                                              cv["u1"], cv["v0"], cv["v1"], cv["w0"], cv["w1"],
                                              c0, c1, order, variant=variant)
        assert rc == 0
        # driver-style exchange (tests/ring2d/test.c:104-105): newest becomes input
        c0, c1 = newest.copy(), other.copy()
    return cv, c0, c1


def main():
    oracle.build(reference=True)
    if not oracle.ref_available("f32"):
        raise SystemExit("reference libraries missing (needs the reference checkout)")
    written = []
    shapes = [(12, 10, 8), (9, 7, 3), (3, 5, 4)]
    for variant in ("f32", "f64"):
        for si, (nx, ny, ns) in enumerate(shapes):
            for order in (1, 2, 3, 4):
                steps = 3 if si == 0 else 1
                case = random_case(nx, ny, ns, seed=100 * si + order)
                cv, newest, other = run_ref(case, order, variant, steps=steps)
                name = f"rand_{nx}x{ny}x{ns}_o{order}_s{steps}_{variant}.npz"
                np.savez_compressed(os.path.join(HERE, name), order=order, steps=steps,
                                    newest=newest, other=other,
                                    **{k: v for k, v in cv.items()})
                written.append(name)
    # The reference's own ring initialisation (tests/init.c:15-103), order 3.
    for variant, (n, m, steps) in (("f32", (16, 3, 20)), ("f64", (16, 3, 20)),
                                   ("f32", (12, 12, 4))):
        t = oracle.ref_test_init(n, m, variant)
        case = dict(u0=t["u"], u1=t["u"], v0=t["v"], v1=t["v"], w0=t["w"], w1=t["w"],
                    c0=t["c0"], dx=t["dx"], dy=t["dy"], ds=t["ds"], dt=t["dt"])
        cv, newest, other = run_ref(case, t["order"], variant, steps=steps)
        name = f"testinit_{n}x{n}x{m}_o{t['order']}_s{steps}_{variant}.npz"
        np.savez_compressed(os.path.join(HERE, name), order=t["order"], steps=steps,
                            newest=newest, other=other, **{k: v for k, v in cv.items()})
        written.append(name)
    print("\n".join(written))


def integer_fixtures():
    """The reference's INTEGER build (real = long).  Its integer scheme can
    divide by zero, where the reference traps: each candidate case is screened
    with the oracle first (over all its steps) and kept only if no division by
    zero occurs and every value stays below 2^31 (far from 64-bit overflow)."""
    oracle.build(reference=True)
    if not oracle.ref_available("i64"):
        raise SystemExit("reference INTEGER library missing (needs the reference checkout)")
    written = []
    for (nx, ny, ns), order, steps in (((9, 7, 5), 1, 2), ((9, 7, 5), 2, 2), ((9, 7, 5), 3, 1),
                                       ((9, 7, 5), 4, 1), ((12, 10, 8), 1, 3),
                                       ((12, 10, 8), 2, 2), ((3, 5, 4), 3, 1)):
        for seed in range(2000):
            case = integer_case(nx, ny, ns, seed=seed, cmax=1000, moving=0.02)
            c0 = case["c0"].copy()
            c1 = np.zeros_like(c0)
            good = True
            for _ in range(steps):
                rc, newest, other = oracle.smolar(case["dx"], case["dy"], case["ds"], case["dt"],
                                                  case["u0"], case["u1"], case["v0"], case["v1"],
                                                  case["w0"], case["w1"], c0, c1, order,
                                                  dtype=np.int64)
                if rc != 0 or max(np.abs(newest).max(), np.abs(other).max()) >= 2 ** 31:
                    good = False
                    break
                c0, c1 = newest.copy(), other.copy()
            if good:
                break
        else:
            raise SystemExit(f"no usable integer case for {nx}x{ny}x{ns} order {order}")
        cv, newest, other = run_ref(case, order, "i64", steps=steps)
        name = f"int_{nx}x{ny}x{ns}_o{order}_s{steps}_i64.npz"
        np.savez_compressed(os.path.join(HERE, name), order=order, steps=steps, seed=seed,
                            newest=newest, other=other, **{k: v for k, v in cv.items()})
        written.append(name)
    print("\n".join(written))


if __name__ == "__main__":
    if sys.argv[1:] == ["integer"]:
        integer_fixtures()
    else:
        main()
