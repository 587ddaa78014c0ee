"""Adjoint of the polychromatic projection with respect to the six float
element volumes: against the FP64 gradient of the oracle and against central
finite differences of the FP64 forward (h = 1e-3 on 64 random voxels); the
two volume loaders against each other."""
import numpy as np
import pytest

import oracle as O
from tests.cases import proj_case, spectrum
from virtualcbct_b200 import Projector

pytestmark = pytest.mark.gpu


def _float_case(seed=0, **kw):
    g, tabs, vol, _ = proj_case("ellipsoid", seed=seed, **kw)
    rng = np.random.default_rng(seed)
    volf = vol.astype(np.float32) * rng.uniform(0.9, 1.1, size=vol.shape).astype(np.float32)
    return g, tabs, volf


def test_float_volume_forward_matches_oracle(cuda):
    import torch
    g, tabs, volf = _float_case(1)
    mu, pdf = spectrum()
    p = Projector(g, *tabs)
    p.set_spectrum(mu, pdf, 1000.0)
    p.load_volume_f32(torch.from_numpy(volf).to(cuda))
    out = p.forward().cpu().numpy()
    ref = O.mbfpa_forward(g, tabs, None, mu, pdf, 1000.0, volf=volf, exact=False, want=("d",))["d"]
    assert np.max(np.abs(out - ref) / ref) <= 1e-5


def test_uint16_and_float_loaders_give_the_same_volume(cuda):
    """Both loaders write the same packed form (float records): a uint16
    volume and the float volume of the same values project bit for bit
    alike, and the adjoint runs on either, with the same gradient."""
    import torch
    g, tabs, vol, _ = proj_case("ellipsoid", seed=3)
    mu, pdf = spectrum()
    pu, pf = Projector(g, *tabs), Projector(g, *tabs)
    for p in (pu, pf):
        p.set_spectrum(mu, pdf, 1000.0)
    pu.load_volume(vol)
    pf.load_volume_f32(torch.from_numpy(vol.astype(np.float32)).to(cuda))
    ou, of = pu.forward(), pf.forward()
    assert torch.equal(ou, of)
    ref = O.mbfpa_forward(g, tabs, vol, mu, pdf, 1000.0, exact=False, want=("d",))["d"]
    assert np.max(np.abs(ou.cpu().numpy() - ref) / ref) <= 1e-5
    resid = torch.from_numpy(np.random.default_rng(7).normal(size=(g.V, g.H, g.W)).astype(np.float32)).to(cuda)
    gu = torch.zeros((g.Z, g.nmat, g.N, g.N), dtype=torch.float32, device=cuda)
    gf = torch.zeros_like(gu)
    pu.adjoint(resid, gu)
    pf.adjoint(resid, gf)
    assert gu.abs().max() > 0
    # float atomics may reduce in another order: equal to FP32 rounding
    assert torch.allclose(gu, gf, rtol=1e-5, atol=1e-6 * gu.abs().max().item())


@pytest.mark.parametrize("seed,zreg,keep", [(0, 0.3, True), (4, 0.3, False), (2, 0.0, True), (2, 0.0, False)])
def test_adjoint_matches_fp64_gradient(cuda, seed, zreg, keep):
    """Both backward forms: path integrals kept from the forward launch, or
    recomputed by a first march (keep_limit = 0)."""
    import torch
    from virtualcbct_b200.autograd import KEEP_LIMIT, project
    g, tabs, volf = _float_case(seed, z_reg=zreg)
    mu, pdf = spectrum()
    rng = np.random.default_rng(100 + seed)
    resid = rng.normal(size=(g.V, g.H, g.W)).astype(np.float32)
    p = Projector(g, *tabs)
    p.set_spectrum(mu, pdf, 1000.0)
    v = torch.from_numpy(volf).to(cuda).requires_grad_(True)
    out = project(v, p, KEEP_LIMIT if keep else 0)
    (out * torch.from_numpy(resid).to(cuda)).sum().backward()
    gpu = v.grad.cpu().numpy().astype(np.float64)
    ref = O.mbfpa_adjoint(g, tabs, volf, mu, pdf, 1000.0, resid.astype(np.float64))
    scale = np.abs(ref).max()
    assert scale > 0
    assert np.abs(gpu - ref).max() <= 2e-4 * scale
    rel = np.linalg.norm(gpu - ref) / np.linalg.norm(ref)
    assert rel <= 1e-5


def test_adjoint_matches_central_finite_differences(cuda):
    """loss = 0.5 * sum (I - target)^2, target from a phantom with +10% Ca/P."""
    import torch
    from virtualcbct_b200.autograd import decomposition_step
    g, tabs, volf = _float_case(7, N=40, Z=12, V=3, W=32, H=28)
    mu, pdf = spectrum()
    tgt_vol = volf.copy()
    tgt_vol[:, 4] *= 1.1
    tgt_vol[:, 5] *= 1.1
    target = O.mbfpa_forward(g, tabs, None, mu, pdf, 1000.0, volf=tgt_vol, exact=False, want=("d",))["d"]
    p = Projector(g, *tabs)
    p.set_spectrum(mu, pdf, 1000.0)
    loss, grad = decomposition_step(torch.from_numpy(volf).to(cuda), torch.from_numpy(target.astype(np.float32)).to(cuda), p)
    grad = grad.cpu().numpy()

    def loss64(v):
        d = O.mbfpa_forward(g, tabs, None, mu, pdf, 1000.0, volf=v, exact=False, want=("d",))["d"]
        return 0.5 * np.sum((d - target) ** 2)

    rng = np.random.default_rng(1234)
    # 64 random voxels with a non-negligible gradient (inside the traversed region)
    cand = np.argwhere(np.abs(grad) > 1e-3 * np.abs(grad).max())
    pick = cand[rng.choice(len(cand), size=64, replace=False)]
    # h = 2^-10 (~1e-3): v +- h is exact in float32 for |v| < 2^14
    h = 2.0 ** -10
    assert np.abs(volf).max() < 2 ** 14
    errs = []
    for idx in map(tuple, pick):
        vp = volf.astype(np.float64).copy(); vm = vp.copy()
        vp[idx] += h; vm[idx] -= h
        fd = (loss64(vp.astype(np.float32)) - loss64(vm.astype(np.float32))) / (2 * h)
        errs.append(abs(fd - grad[idx]) / max(abs(grad[idx]), 1e-30))
    assert np.median(errs) <= 1e-3 and np.max(errs) <= 2e-2


def test_forward_state_is_forward_plus_path_integrals(cuda):
    import torch
    g, tabs, volf = _float_case(3)
    mu, pdf = spectrum()
    p = Projector(g, *tabs)
    p.set_spectrum(mu, pdf, 1000.0)
    p.load_volume_f32(torch.from_numpy(volf).to(cuda))
    out, L = p.forward_state()
    assert torch.equal(out, p.forward())
    assert torch.equal(L, p.path_integrals())
    rng = np.random.default_rng(7)
    go = torch.from_numpy(rng.normal(size=(g.V, g.H, g.W)).astype(np.float32)).to(cuda)
    a = p.adjoint(go).double()
    b = p.adjoint_state(L, go).double()
    # the same contributions; only the order of the atomic additions differs
    assert (a - b).abs().max().item() <= 1e-5 * a.abs().max().item()


@pytest.mark.parametrize("strips", [2, 3, 5])
def test_adjoint_row_strips_match_fp64_gradient(cuda, monkeypatch, strips):
    """The adjoint scattered in strips of volume rows (one launch per strip,
    each marching only the iterations that can reach its rows; by default
    only for gradient planes above 0.5 GB) against the FP64 gradient, with
    kept path integrals, including the z = 0 boundary plane (z_reg = 0)."""
    import torch
    from virtualcbct_b200.autograd import project
    monkeypatch.setenv("VCBCT_ADJ_STRIPS", str(strips))
    g, tabs, volf = _float_case(3, z_reg=0.0)
    mu, pdf = spectrum()
    resid = np.random.default_rng(11).normal(size=(g.V, g.H, g.W)).astype(np.float32)
    p = Projector(g, *tabs)
    p.set_spectrum(mu, pdf, 1000.0)
    v = torch.from_numpy(volf).to(cuda).requires_grad_(True)
    out = project(v, p, 1 << 40)                      # path integrals kept
    (out * torch.from_numpy(resid).to(cuda)).sum().backward()
    gpu = v.grad.cpu().numpy().astype(np.float64)
    ref = O.mbfpa_adjoint(g, tabs, volf, mu, pdf, 1000.0, resid.astype(np.float64))
    assert np.linalg.norm(gpu - ref) / np.linalg.norm(ref) <= 1e-5
