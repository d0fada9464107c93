"""CPU checks of the benchmark's accuracy helpers (no GPU): the error
breakdown, the local-extremum test, the half-ulp perturbation, and that the
reference arm's workload loader does not load the product library."""
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    import bench  # the repository root is on sys.path (conftest.py)
    return bench


def test_error_breakdown_shares():
    b = _bench()
    ref = np.ones((4, 5, 6))
    a = ref.copy()
    a[2, 3, 1] += 0.3   # column x = 1
    a[1, 2, 4] += 0.4   # inside
    out, e = b.error_breakdown(a, ref, float(np.linalg.norm(ref)))
    assert np.isclose(out["rel_l2"], 0.5 / np.linalg.norm(ref))
    assert np.isclose(out["max_abs"], 0.4)
    assert np.isclose(out["share_column_x1"], 0.09 / 0.25)
    assert np.isclose(out["rel_l2_without_x_le_2"], 0.4 / np.linalg.norm(ref))
    assert out["negative_cells"] == 0 and e.size == ref.size


def test_local_extremum_and_perturbation():
    b = _bench()
    c = np.zeros((5, 5, 5))
    c[2, 2, 2] = 1.0
    c[2, 2, 3] = 0.5
    idx = np.ravel_multi_index(([2, 2, 0], [2, 2, 0], [2, 3, 0]), c.shape)
    ext = b.local_extremum(c, idx)
    assert list(ext) == [True, False, False]  # max; not an extremum; shell cell
    p = b.half_ulp_perturbed(np.full((3, 4, 5), 2.0))
    assert np.all(np.abs(p / 2.0 - 1.0) <= 2.0 ** -24)
    assert not np.array_equal(p, np.full_like(p, 2.0))


def test_reference_arm_loads_workloads_without_the_library():
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import bench\n"
        "w = bench._workloads_module().roofline(16, 12, 6)\n"
        "assert w['c0'].shape == (6, 12, 16)\n"
        "maps = open('/proc/self/maps').read()\n"
        "assert 'libmpdata_b200' not in maps, 'product library mapped'\n"
        "assert 'mpdata_b200' not in sys.modules\n" % ROOT)
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr


def test_kernel_option_keeps_the_forms_the_kernel_runs():
    """--kernel 1 (one kernel per reference routine) keeps only the IEEE form
    (approx_div needs the fused kernels) and labels the roofline kernel."""
    code = ("import bench; bench._set_kernel(1); "
            "print([n for n, _ in bench.FORMS], bench.FORMS[0][1]['kernel'], "
            "bench.KERNEL_OF_FORM['plain'].split()[0])")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                         check=True).stdout.split()
    assert out == ["['plain']", "1", "k_antidiff"]
    code = ("import bench; bench._set_kernel(2); print(len(bench.FORMS), "
            "all(o['kernel'] == 2 for _, o in bench.FORMS))")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                         check=True).stdout.split()
    assert out == ["3", "True"]


def test_check_courant_option_reaches_every_form():
    code = ("import bench; bench._add_form_options(check_courant=True); "
            "print(all(o.get('check_courant') for _, o in bench.FORMS), len(bench.FORMS))")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                         check=True).stdout.split()
    assert out == ["True", "3"]
