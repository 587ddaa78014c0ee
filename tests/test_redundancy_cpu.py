"""Redundancy weights of an offset (half-fan) detector (no reference
counterpart; the FDK applies them to -log p with redundancy = 1):
the library's weights against a restatement of their formula, and the
property they exist for -- a ray and its conjugate weigh 2 together."""
import numpy as np
import pytest

from virtualcbct_b200 import FdkGeometry, VcbctError, redundancy_weights


def _restated(g, xs):
    """w = 2 sin^2(pi/4 (1 + x)), x = side * u / u0, clamped to [0, 2], where
    u is the column's position at the isocentre (filterSinogram.cpp:86 centre
    convention) and u0 the half-width of the band seen from both sides."""
    W = g.W
    pitch = g.piso * g.mpn / W
    px = g.pdet * g.mpn / W
    w = np.ones((g.V, W))
    for v in range(g.V):
        xcs = -W / 2.0 - xs[v] / px - 1
        umin, umax = xcs * pitch, (xcs + W - 1) * pitch
        u0 = min(-umin, umax)
        if not u0 > 0:
            continue
        side = 1.0 if umax >= -umin else -1.0
        x = side * (xcs + np.arange(W)) * pitch / u0
        w[v] = np.where(x >= 1, 2.0, np.where(x <= -1, 0.0, 2.0 * np.sin(np.pi / 4 * (1 + np.clip(x, -1, 1))) ** 2))
    return w


@pytest.mark.parametrize("W,shift", [(400, 16.0), (400, -16.0), (256, 7.5), (64, 0.0)])
def test_weights_match_their_formula(W, shift):
    g = FdkGeometry(W=W, V=5, redundancy=1)
    xs = np.full(g.V, shift) + np.arange(g.V) * 0.25
    w = redundancy_weights(g, xs)
    assert w.shape == (g.V, W) and w.dtype == np.float32
    assert np.abs(w - _restated(g, xs)).max() <= 1e-6
    assert w.min() >= 0.0 and w.max() <= 2.0


def test_a_ray_and_its_conjugate_weigh_two():
    """Config-2 detector: 400 columns offset by 160 pixels (xshift 16 x 10 px).
    The conjugate of the ray at lateral position u lies at -u; where both are
    on the detector their weights sum to 2, and where only one is, it weighs 2."""
    g = FdkGeometry(W=400, V=1, redundancy=1)
    w = redundancy_weights(g, np.array([16.0]))[0].astype(np.float64)
    pitch = g.piso * g.mpn / g.W
    px = g.pdet * g.mpn / g.W
    u = (-g.W / 2.0 - 16.0 / px - 1 + np.arange(g.W)) * pitch
    lo, hi = u.min(), u.max()
    inside = (-u >= lo) & (-u <= hi)
    w_conj = np.interp(-u[inside], u, w)
    assert np.abs(w[inside] + w_conj - 2.0).max() <= 2e-3  # linear interpolation between columns
    assert np.all(w[~inside] == 2.0)
    assert inside.sum() > 0 and (~inside).sum() > 0
    # monotone from the short edge (weight 0) to the long side (weight 2)
    side = 1 if hi >= -lo else -1
    ws = w if side > 0 else w[::-1]
    assert np.all(np.diff(ws) >= -1e-7) and ws[0] == 0.0 and ws[-1] == 2.0


def test_weights_reject_bad_arguments():
    g = FdkGeometry(W=1, V=2)
    with pytest.raises(VcbctError):
        redundancy_weights(g, np.zeros(2))
    with pytest.raises(ValueError):
        redundancy_weights(FdkGeometry(V=3), np.zeros(2))
