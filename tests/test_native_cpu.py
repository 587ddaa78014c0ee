"""CPU-side checks of the C ABI library: it loads without a GPU and exports
every entry point include/vcbct.h declares (the reference-named C++-linkage
entry points of include/vcbct_reference.h are checked in test_dropin_cpu.py);
argument validation fails with a status (no CUDA call is made on these
paths)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from virtualcbct_b200 import _native as N
from virtualcbct_b200 import ProjGeometry, trig_tables, attenuation_table

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _declared_symbols():
    text = open(os.path.join(ROOT, "include", "vcbct.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set()
    for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
        name = m.group(1)
        if name in ("if", "sizeof", "defined"):
            continue
        names.add(name)
    # keep only function declarations (type names are not followed by '(')
    return {n for n in names if not n.startswith("VCBCT_")}


def test_library_loads_and_exports_every_declared_symbol():
    L = N.lib()
    declared = _declared_symbols()
    assert "vcbct_reprojectionOnGPU" in declared and "vcbct_projector_forward" in declared
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing
    assert set(N.SIGNATURES) == declared


def test_version_and_error_strings():
    L = N.lib()
    assert b"sm_100a" in L.vcbct_version()


def test_create_rejects_bad_geometry():
    L = N.lib()
    g = ProjGeometry(N=0, Z=4, s=0.1, step=0.1, W=8, H=8, V=2).to_c()
    h = C.c_void_p()
    t = np.zeros(2)
    p = t.ctypes.data_as(C.POINTER(C.c_double))
    rc = L.vcbct_projector_create(C.byref(g), p, p, p, p, C.byref(h))
    assert rc == 1 and h.value is None
    assert b"positive" in L.vcbct_last_error()
    g = ProjGeometry(N=8, Z=4, s=0.1, step=0.1, W=8, H=8, V=2, nmat=9).to_c()
    assert L.vcbct_projector_create(C.byref(g), p, p, p, p, C.byref(h)) == 3


def test_trig_tables_match_oracle():
    import oracle as O
    ang = np.deg2rad(np.array([-170.0001, -10.5, 33.0, 179.9]))
    xs = np.array([0.0, 1.6, -0.3, 0.05])
    ys = np.array([0.0, 0.1, 0.0, -0.2])
    a = trig_tables(400, 400, ang, xs, ys)
    b = O.trig_tables(400, 400, ang, xs, ys, 0.05, 800.0)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_attenuation_table_errors():
    with pytest.raises(N.VcbctError):
        attenuation_table("/nonexistent.csv", "/nonexistent", 6)
