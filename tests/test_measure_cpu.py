"""The bench-only gather probe library: built apart from the product library,
exports its entry points, and rejects a bad probe kind without a GPU."""
import ctypes as C
import os
import subprocess

import pytest

import measure

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def test_probe_is_not_in_the_product_library():
    out = subprocess.run(["nm", "-D", "--defined-only", os.path.join(ROOT, "virtualcbct_b200", "libvcbct.so")],
                         capture_output=True, text=True, check=True).stdout
    assert "probe" not in out


def test_probe_library_rejects_bad_kind():
    L = measure._lib()
    r = C.c_double()
    assert L.gather_probe_run(4, C.byref(r), None) == 1
    assert b"kind" in L.gather_probe_error()
    with pytest.raises(RuntimeError):
        measure.probe_gather(-1)
