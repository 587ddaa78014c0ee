"""vcbct_projector_project (host volume in, host projections out, upload
overlapped with the projection by detector row band) against the two-call
form vcbct_projector_load_volume + vcbct_projector_forward: bitwise equal.

A band launched before the slices it reads are uploaded would read the
previous volume's values, so every case first loads a different volume
(large values everywhere) and checks that none of it shows through."""
import numpy as np
import pytest

from tests.cases import proj_case, spectrum
from virtualcbct_b200 import Projector, phantoms

pytestmark = pytest.mark.gpu

CASES = [
    # kind, geometry overrides
    ("ellipsoid", dict(seed=3)),
    ("random", dict(seed=1, z_reg=0.0)),                        # central row in a slice plane
    ("random", dict(seed=2, z_reg=1.7, H=70, Z=21)),            # off-centre source, ragged bands/slabs
    ("water", dict(N=128, Z=40, s=0.1, W=96, H=100, V=12, xshift=3.0)),
    ("random", dict(seed=4, N=96, Z=64, s=0.15, step=0.12, W=64, H=130, V=6, dpn=900.0)),  # steep cone
    ("random", dict(seed=6, H=33, V=3)),                        # fewer views than the last band's chunks
]


def _pair(kind, kw, pinned):
    import torch
    g, tabs, vol, _ = proj_case(kind, **kw)
    mu, pdf = spectrum()
    p = Projector(g, *tabs)
    p.set_spectrum(mu, pdf, 1000.0)
    p.load_volume(vol)
    ref = np.empty((g.V, g.H, g.W), np.float32)
    p.forward(ref)
    # a different volume resident first, then the one-call form
    p.load_volume(np.full_like(vol, 4000))
    if pinned:
        out = torch.empty((g.V, g.H, g.W), dtype=torch.float32).pin_memory().numpy()
    else:
        out = np.empty((g.V, g.H, g.W), np.float32)
    out[...] = np.nan
    p.project(vol, out)
    return ref, out, p, vol


@pytest.mark.parametrize("pinned", [True, False])
@pytest.mark.parametrize("kind,kw", CASES)
def test_project_equals_load_and_forward(cuda, kind, kw, pinned):
    ref, out, p, vol = _pair(kind, kw, pinned)
    assert np.array_equal(out, ref)
    # the volume stays loaded: a device forward afterwards gives the same
    again = np.empty_like(ref)
    p.forward(again)
    assert np.array_equal(again, ref)


@pytest.mark.parametrize("pinned", [True, False])
def test_project_twice_and_with_noise(cuda, pinned):
    """Noise counters follow the global view index, also in the last band's
    view chunks (page-locked output)."""
    import torch
    g, tabs, vol, _ = proj_case("random", seed=5, N=96, Z=30, W=64, H=72, V=8)
    vol2 = phantoms.random_volume(96, 30, seed=6, hi=500)
    mu, pdf = spectrum()
    p = Projector(g, *tabs)
    p.set_spectrum(mu, pdf, 1000.0)
    p.set_noise(5.0e4, 6.0e4, seed=11)
    outs = []
    for v in (vol, vol2, vol):
        p.load_volume(v)
        ref = np.empty((g.V, g.H, g.W), np.float32)
        p.forward(ref)
        out = torch.empty((g.V, g.H, g.W), dtype=torch.float32).pin_memory().numpy() if pinned else None
        out = p.project(v, out)
        assert np.array_equal(out, ref)
        outs.append(out)
    assert np.array_equal(outs[0], outs[2]) and not np.array_equal(outs[0], outs[1])


def test_project_needs_spectrum(cuda):
    import virtualcbct_b200 as vc
    g, tabs, vol, _ = proj_case("random", seed=0)
    p = Projector(g, *tabs)
    with pytest.raises(vc.VcbctError, match="spectrum"):
        p.project(vol)
