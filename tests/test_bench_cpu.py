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


def test_effective_update_count_matches_a_direct_count():
    """The backprojection's effective voxel-view updates (the denominator of
    its gather-roof fraction): the per-view slice-range formula of
    bench.bp_update_counts against a direct per-voxel test of the detector
    column and row, on a small half-fan geometry."""
    fg = FdkGeometry(W=16, H=12, V=12, N=21, Z=14, zstart=-10, step=1.5, scale=1.0)
    ang = np.deg2rad(-180.0001 + np.arange(fg.V) * 30.0)
    xs = np.full(fg.V, 4.0)  # an offset detector (x10 px)
    n_all, n_mask, n_eff = bench.bp_update_counts(fg, ang, xs)
    N, Z, W, H = fg.N, fg.Z, fg.W, fg.H
    R = (N - 1) / 2.0
    y, x = np.mgrid[0:N, 0:N].astype(np.float64)
    m = (y - R) ** 2 + (x - R) ** 2 <= R * R
    cp = N / 2.0 - 0.5
    xx, yy = ((x - cp) * fg.scale)[m], (-(y - cp) * fg.scale)[m]
    pitch = fg.piso * fg.mpn / W
    px = fg.pdet * fg.mpn / W
    zz = fg.zstart + np.arange(Z) * fg.step
    eff = 0
    for th in range(fg.V):
        cs, sn = np.cos(ang[th]), np.sin(ang[th])
        g = 1.0 / ((1.0 - (-xx * sn + yy * cs) / fg.sad) * pitch)
        uu = np.floor((W // 2) + xs[th] / px - 0.5 + (xx * cs + yy * sn) * g)
        row = np.floor((H // 2) + zz[None, :] * g[:, None])
        ok = ((uu >= 0) & (uu <= W - 1))[:, None] & (row >= 0) & (row <= H - 1)
        eff += int(ok.sum())
    assert n_all == N * N * Z * fg.V and n_mask == int(m.sum()) * Z * fg.V
    assert 0 < eff < n_mask
    assert abs(n_eff - eff) <= 1e-3 * eff
