"""`bench.py`'s CPU baseline of the FDK: the reference's filterSinogram and
reconstructImage timed on a view sample and extrapolated to the whole stack."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
import oracle as O  # noqa: E402
from virtualcbct_b200 import FdkGeometry  # noqa: E402


@pytest.mark.skipif(not O.have_reference(), reason="reference objects not built")
def test_fdk_cpu_baseline_times_the_reference_on_a_sample():
    fg = FdkGeometry(W=64, H=64, V=20, N=27, Z=4, zstart=-1, step=0.2, scale=0.1)
    ang = np.deg2rad(np.arange(fg.V) * 18.0 - 180.0001)
    xs = np.zeros(fg.V)
    views = np.arange(0, fg.V, 5)
    rng = np.random.default_rng(3)
    proj = rng.uniform(0.2, 1.0, size=(len(views), fg.H, fg.W)).astype(np.float32)
    filt = rng.normal(size=(len(views), fg.H, fg.W)).astype(np.float32)
    r = bench.fdk_cpu_baseline(fg, ang, xs, views, proj, filt)
    assert r["kind"] == "reference" and r["cores"] >= 1
    assert r["filter_ms"] > 0 and r["bp_ms"] > 0
    assert r["bp_gups"] == pytest.approx(fg.N * fg.N * fg.Z * fg.V / (r["bp_ms"] * 1e-3) / 1e9)
    assert f"on {len(views)} of {fg.V} views" in r["sample"]


def test_fdk_cpu_baseline_is_never_fatal():
    fg = FdkGeometry(W=64, H=64, V=20, N=27, Z=4)
    # no projections: the helper reports the failure instead of raising
    r = bench.fdk_cpu_baseline(fg, np.zeros(fg.V), np.zeros(fg.V), np.arange(3), None, None)
    assert r["kind"] == "reference" and r["value"] is None
    assert r["sample"].startswith("unavailable")
