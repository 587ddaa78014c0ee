"""Element counts other than six (the reference's num_material is a run-time
argument of initializeGPU; this library takes 1 to VCBCT_MAX_MATERIALS = 8):
projections, path integrals and the adjoint against the FP64 oracle, and
batches that mix counts against per-phantom launches."""
import numpy as np
import pytest

import oracle as O
from tests.cases import spectrum
from virtualcbct_b200 import Batch, Projector, ProjGeometry, phantoms, trig_tables

pytestmark = pytest.mark.gpu

COUNTS = [1, 2, 4, 5, 7, 8]


def _mu(nmat):
    """[nmat][NE] attenuation rows: the six elements' rows repeated, each
    repeat scaled by another factor, so that every row differs."""
    mu6, pdf = spectrum()
    mu = np.stack([mu6[k % 6] * np.float32(1.0 + 0.15 * (k // 6)) for k in range(nmat)])
    return mu.astype(np.float32), pdf


def _case(nmat, seed=0, N=40, Z=12, s=0.25, step=0.5, W=36, H=40, V=3, z_reg=0.3):
    g = ProjGeometry(N=N, Z=Z, s=s, step=step, W=W, H=H, V=V, dpn=480.0, z_reg=z_reg, nmat=nmat)
    ang = np.deg2rad(phantoms.view_angles(V))
    tabs = trig_tables(W, H, ang, np.zeros(V), np.zeros(V), g.pdet, g.dpn)
    vol = phantoms.random_volume(N, Z, nmat=nmat, seed=seed, hi=400 // nmat + 50)
    return g, tabs, vol


@pytest.mark.parametrize("nmat", COUNTS)
def test_uint16_forward_and_path_integrals(cuda, nmat):
    g, tabs, vol = _case(nmat, seed=nmat)
    mu, pdf = _mu(nmat)
    p = Projector(g, *tabs)
    p.set_spectrum(mu, pdf, 1000.0)
    p.load_volume(vol)
    out = np.empty((g.V, g.H, g.W), np.float32)
    p.forward(out)
    ref = O.mbfpa_forward(g, tabs, vol, mu, pdf, 1000.0, exact=True, want=("d",))["d"]
    assert np.isfinite(out).all()
    assert np.max(np.abs(out - ref) / ref) <= 1e-5
    L = p.path_integrals().cpu().numpy()
    ref_L = O.mbfpa_forward(g, tabs, vol, mu, pdf, 1000.0, exact=False, want=("L",))["L"]
    assert L.shape == (g.V, g.H, g.W, nmat)
    assert np.abs(ref_L).max() > 0
    assert np.abs(L - ref_L).max() <= 2e-5 * np.abs(ref_L).max()


@pytest.mark.parametrize("nmat", COUNTS)
def test_float_forward_state(cuda, nmat):
    import torch
    g, tabs, vol = _case(nmat, seed=10 + nmat)
    volf = vol.astype(np.float32) * np.random.default_rng(nmat).uniform(0.9, 1.1, vol.shape).astype(np.float32)
    mu, pdf = _mu(nmat)
    p = Projector(g, *tabs)
    p.set_spectrum(mu, pdf, 1000.0)
    p.load_volume_f32(torch.from_numpy(volf).to(cuda))
    out, L = p.forward_state()
    ref = O.mbfpa_forward(g, tabs, None, mu, pdf, 1000.0, volf=volf, exact=False, want=("d", "L"))
    assert np.abs(ref["L"]).max() > 0
    assert np.max(np.abs(out.cpu().numpy() - ref["d"]) / ref["d"]) <= 1e-5
    assert np.abs(L.cpu().numpy() - ref["L"]).max() <= 2e-5 * np.abs(ref["L"]).max()


@pytest.mark.parametrize("nmat,keep", [(1, True), (2, False), (5, True), (7, False), (8, True), (8, False)])
def test_adjoint_matches_fp64_gradient(cuda, nmat, keep):
    import torch
    from virtualcbct_b200.autograd import KEEP_LIMIT, project
    g, tabs, vol = _case(nmat, seed=20 + nmat, z_reg=0.0)
    volf = vol.astype(np.float32) * np.random.default_rng(nmat).uniform(0.9, 1.1, vol.shape).astype(np.float32)
    mu, pdf = _mu(nmat)
    resid = np.random.default_rng(30 + nmat).normal(size=(g.V, g.H, g.W)).astype(np.float32)
    p = Projector(g, *tabs)
    p.set_spectrum(mu, pdf, 1000.0)
    v = torch.from_numpy(volf).to(cuda).requires_grad_(True)
    out = project(v, p, KEEP_LIMIT if keep else 0)
    (out * torch.from_numpy(resid).to(cuda)).sum().backward()
    gpu = v.grad.cpu().numpy().astype(np.float64)
    ref = O.mbfpa_adjoint(g, tabs, volf, mu, pdf, 1000.0, resid.astype(np.float64))
    assert gpu.shape == (g.Z, nmat, g.N, g.N)
    assert np.linalg.norm(gpu - ref) / np.linalg.norm(ref) <= 1e-5


def test_batch_mixing_element_counts_equals_plain_launches(cuda):
    """A batch whose items hold 2, 6 and 8 elements runs the eight-element
    kernels for all of them; an item's attenuation rows beyond its element
    count are zero, so every item's projection is bitwise its own launch's."""
    import torch
    ps = []
    for nmat, seed in ((2, 1), (6, 2), (8, 3)):
        g, tabs, vol = _case(nmat, seed=seed, N=48, Z=10, V=2)
        mu, pdf = _mu(nmat)
        p = Projector(g, *tabs)
        p.set_spectrum(mu, pdf, 1000.0)
        p.load_volume(torch.from_numpy(vol.view(np.int16)).to(cuda))
        ps.append(p)
    plain = [p.forward().cpu().numpy() for p in ps]
    b = Batch()
    outs = [b.add(p) for p in ps]
    for strategy in (0, 1, 2):
        b.configure(strategy, 4)
        for o in outs:
            o.fill_(float("nan"))
        b.forward(use_graph=False)
        torch.cuda.synchronize()
        for o, ref in zip(outs, plain):
            assert np.array_equal(o.cpu().numpy(), ref), strategy
