"""C-ABI checks that need no GPU: the library loads, exports every entry point
the public header declares, and rejects bad arguments before touching CUDA."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "mpdata_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if not n.startswith("_")))


def test_header_declares_reference_entry_points():
    names = declared_functions()
    for n in ("smolar", "smolar_f64", "msmolar", "msmolar_gather", "msmolar_free",
              "mpdata_create", "mpdata_step", "mpdata_destroy"):
        assert n in names


def test_library_exports_every_declared_symbol():
    import mpdata_b200
    lib = mpdata_b200.library()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_library_is_in_tree_and_native():
    import mpdata_b200
    assert os.path.dirname(mpdata_b200.LIB_PATH) == os.path.join(ROOT, "mpdata_b200")
    assert open(mpdata_b200.LIB_PATH, "rb").read(4) == b"\x7fELF"


def _args(n=(5, 4, 3), dtype=np.float32):
    nx, ny, ns = n
    z = lambda *s: np.zeros(s, dtype)
    return dict(dx=z(nx), dy=z(ny), ds=z(ns), u=z(ns, ny, nx), c0=z(ns, ny, nx), c1=z(ns, ny, nx))


def test_smolar_rejects_small_grid_without_gpu():
    import mpdata_b200 as m
    a = _args((2, 4, 3))
    with pytest.raises(m.MpdataError) as e:
        m.smolar(2, 4, 3, a["dx"], a["dy"], a["ds"], 1.0, *([a["u"]] * 6), a["c0"], a["c1"],
                 order=2)
    assert e.value.code == -1 and ">= 3" in str(e.value)


def test_smolar_rejects_negative_order_without_gpu():
    import mpdata_b200 as m
    a = _args()
    with pytest.raises(m.MpdataError) as e:
        m.smolar(5, 4, 3, a["dx"], a["dy"], a["ds"], 1.0, *([a["u"]] * 6), a["c0"], a["c1"],
                 order=-1)
    assert e.value.code == -1


def test_smolar_order_zero_only_exchanges_pointers():
    """The reference runs no pass for order 0 but still swaps *c0/*c1
    (core/src/smolar.c:46-58); no GPU work is needed for that."""
    import mpdata_b200 as m
    a = _args()
    a["c0"][:] = 1.0
    c0, c1 = m.smolar(5, 4, 3, a["dx"], a["dy"], a["ds"], 1.0, *([a["u"]] * 6), a["c0"],
                      a["c1"], order=0)
    assert c0 is a["c1"] and c1 is a["c0"]
    assert (c1 == 1.0).all()


def test_smolar_i64_argument_checks_without_gpu():
    """The INTEGER-build twin checks its arguments before any CUDA call, and
    order 0 only exchanges the pointers, as the float entries do."""
    import mpdata_b200 as m
    a = _args(dtype=np.int64)
    with pytest.raises(m.MpdataError) as e:
        m.smolar(5, 4, 2, a["dx"], a["dy"], a["ds"][:2], 1, *([a["u"]] * 6), a["c0"], a["c1"],
                 order=2, dtype=np.int64)
    assert e.value.code == -1
    with pytest.raises(m.MpdataError) as e:
        m.smolar(5, 4, 3, a["dx"], a["dy"], a["ds"], 1, *([a["u"]] * 6), a["c0"], a["c1"],
                 order=-1, dtype=np.int64)
    assert e.value.code == -1
    a["c0"][:] = 7
    c0, c1 = m.smolar(5, 4, 3, a["dx"], a["dy"], a["ds"], 1, *([a["u"]] * 6), a["c0"], a["c1"],
                      order=0, dtype=np.int64)
    assert c0 is a["c1"] and c1 is a["c0"] and (c1 == 7).all()


def test_create_rejects_bad_arguments_without_gpu():
    import mpdata_b200 as m
    for kw in (dict(nx=2, ny=5, ns=5, order=2), dict(nx=5, ny=5, ns=5, order=0)):
        with pytest.raises(m.MpdataError) as e:
            m.Solver(kw["nx"], kw["ny"], kw["ns"], order=kw["order"])
        assert e.value.code == -1
    with pytest.raises(m.MpdataError):
        m.Solver(5, 5, 5, order=2, dtype=np.float64, precision_form=True)


def test_options_struct_layout_matches_header():
    import mpdata_b200 as m
    text = open(HEADER).read()
    body = re.search(r"typedef struct mpdata_options \{(.*?)\} mpdata_options;", text, re.S).group(1)
    fields = re.findall(r"int\s+(\w+);", body)
    assert fields == [f for f, _ in m.Options._fields_]


def test_msmolar_free_accepts_null_state():
    import mpdata_b200 as m
    st = m.MsmolarState()
    st.free()
    assert st.desc.value is None
