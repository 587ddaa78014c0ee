"""Detector noise: the forward kernel's Gaussian count noise and the
reference-unit gaussiannoise kernel have the model's distribution, are
reproducible for a seed and independent of launch shape and output path."""
import ctypes as C

import numpy as np
import pytest

from tests.cases import proj_case, spectrum
from virtualcbct_b200 import Projector
from virtualcbct_b200 import _native as N

pytestmark = pytest.mark.gpu


def _projector(cuda):
    import torch
    g, tabs, vol, _ = proj_case("ellipsoid", seed=2, V=6, W=64, H=48)
    mu, pdf = spectrum()
    p = Projector(g, *tabs)
    p.set_spectrum(mu, pdf, 1000.0)
    p.load_volume(torch.from_numpy(vol.view(np.int16)).to(cuda))
    return g, p


def test_forward_count_noise_statistics_and_reproducibility(cuda):
    import torch
    g, p = _projector(cuda)
    clean = p.forward().double()
    i0 = 1.0e5
    p.set_noise(i0, max_counts=1.0e9, seed=42)
    a = p.forward().double()
    b = p.forward().double()
    assert torch.equal(a, b)                               # same seed: same draws
    host = np.empty((g.V, g.H, g.W), np.float32)
    p.forward(host)                                        # view-chunked host path
    assert np.array_equal(host, a.float().cpu().numpy())
    n = i0 * clean
    z = ((a * i0 - n) / n.sqrt()).flatten()
    z = z[n.flatten() > 100]
    m, s = z.mean().item(), z.std().item()
    k = z.numel()
    assert abs(m) < 5.0 / k ** 0.5 and abs(s - 1.0) < 0.05
    p.set_noise(i0, max_counts=1.0e9, seed=43)
    assert not torch.equal(p.forward().double(), a)        # another seed: other draws
    p.set_noise(0.0)
    assert torch.equal(p.forward().double(), clean)        # off again
    p.set_noise(i0, max_counts=0.5 * i0, seed=42)
    c = p.forward()
    assert c.max().item() <= 0.5 + 1e-7 and c.min().item() >= 0.0   # clamped counts


def test_reference_unit_gaussian_noise(cuda):
    import torch
    maxv = 65535.0
    n0 = 20000.0
    x = torch.full((1 << 20,), maxv - n0, dtype=torch.float32, device=cuda)
    y = x.clone()
    N.check(N.lib().vcbct_gaussian_noise(C.c_void_p(y.data_ptr()), y.numel(), maxv, 7, 1, None))
    counts = (maxv - y.double())
    z = (counts - n0) / n0 ** 0.5
    assert abs(z.mean().item()) < 5.0 / y.numel() ** 0.5 and abs(z.std().item() - 1.0) < 0.01
    y2 = x.clone()
    N.check(N.lib().vcbct_gaussian_noise(C.c_void_p(y2.data_ptr()), y2.numel(), maxv, 7, 1, None))
    assert torch.equal(y, y2)
    # a stack that is not 16-byte aligned (the per-pixel path) gets the same draws
    big = torch.empty(1 + 1001, dtype=torch.float32, device=cuda)
    a = x[:1001].clone()
    big[1:] = a
    mis = big[1:]
    N.check(N.lib().vcbct_gaussian_noise(C.c_void_p(a.data_ptr()), a.numel(), maxv, 9, 1, None))
    N.check(N.lib().vcbct_gaussian_noise(C.c_void_p(mis.data_ptr()), mis.numel(), maxv, 9, 1, None))
    assert torch.equal(a, mis)
    # values whose count is 0: p stays at max; counts above max clamp p to 0
    e = torch.tensor([maxv, -1.0e6], dtype=torch.float32, device=cuda)
    N.check(N.lib().vcbct_gaussian_noise(C.c_void_p(e.data_ptr()), 2, maxv, 1, 1, None))
    assert e[0].item() == maxv and e[1].item() == 0.0


@pytest.mark.parametrize("i0", [4.0, 3.0e4])
def test_forward_poisson_counts(cuda, i0):
    """Poisson counts in the epilogue: integer counts, reproducible, mean and
    variance n; at low counts (the multiplication sampler) the numbers of
    zero and one counts match sum exp(-n) and sum n exp(-n); at high counts
    (the PTRS sampler) the skewness matches 1 / sqrt(n)."""
    import torch
    g, p = _projector(cuda)
    clean = p.forward().double()
    p.set_noise(i0, max_counts=1.0e12, seed=5, model="poisson")
    a = p.forward().double()
    assert torch.equal(a, p.forward().double())
    n = (i0 * clean).flatten()
    m = (i0 * a).flatten()
    assert float((m - m.round()).abs().max()) <= 1e-6 * float(m.max()) + 1e-4   # whole counts
    m = m.round()
    keep = n > 0.05
    n, m = n[keep], m[keep]
    k = n.numel()
    z = (m - n) / n.sqrt()
    assert abs(z.mean().item()) < 5.0 / k ** 0.5 and abs(z.std().item() - 1.0) < 0.03
    if i0 < 10:
        for c, pc in ((0, torch.exp(-n)), (1, n * torch.exp(-n))):
            got = float((m == c).sum())
            want = float(pc.sum())
            sd = float((pc * (1 - pc)).sum()) ** 0.5
            assert abs(got - want) < 5 * sd + 1, (c, got, want, sd)
    else:
        skew = ((m - n) ** 3 / n ** 1.5).mean().item()          # E = 1 / sqrt(n) per pixel
        assert abs(skew - (1.0 / n.sqrt()).mean().item()) < 6.0 * (15.0 / k) ** 0.5
    p.set_noise(0.0)
    assert torch.equal(p.forward().double(), clean)
