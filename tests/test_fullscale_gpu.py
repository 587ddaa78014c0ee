"""The full-scale decomposition workload at its real size: six FP32 element
volumes 512x512x400 (0.5 x 0.5 x 1 mm) of a synthetic ellipsoid phantom, 720
views of an 800x800 detector (0.5 mm), a 111-bin 120 kV spectrum; gradient
steps of least-squares material decomposition against projections of the
phantom with bone Ca and P scaled by 1.1 (the backward pass reads the
per-ray path integrals kept from the forward launch, 11 GB, and recomputes
each ray's spectral state from them; the re-marching form, for when they do
not fit, gives the same gradient); then FDK of the final projections to
512x512x400 short.

At this size the FP64 oracle covers samples: 1024 rays of two views for the
projection, two whole views for the ramp filter, two slices for the
backprojection; the gradient is checked by a size-independent property, the
central difference of the loss along a direction against <grad, direction>.
One of the workload's four phantoms is run (the others differ only in the
seed)."""
import os

import numpy as np
import pytest

import oracle as O
from virtualcbct_b200 import (FILTER_BF16X3, Fdk, FdkGeometry, Projector, ProjGeometry, attenuation_table,
                              phantoms, trig_tables)

pytestmark = pytest.mark.gpu

DATA = os.path.join(os.path.dirname(__file__), "..", "virtualcbct_b200", "data")


def _loss(pred, target):
    """0.5 * sum (pred - target)^2 in FP64, a view block at a time."""
    tot = 0.0
    for v0 in range(0, pred.shape[0], 90):
        tot += 0.5 * float(((pred[v0:v0 + 90] - target[v0:v0 + 90]).double() ** 2).sum())
    return tot


def test_fullscale_decomposition_and_fdk(cuda):
    import torch
    from virtualcbct_b200.autograd import decomposition_step, project
    g = ProjGeometry(N=512, Z=400, s=0.05, step=0.1, W=800, H=800, V=720)
    ang = np.deg2rad(phantoms.view_angles(g.V))
    tabs = trig_tables(g.W, g.H, ang, np.zeros(g.V), np.zeros(g.V), g.pdet, g.dpn)
    mu, pdf = attenuation_table(os.path.join(DATA, "spectrum_kramers120_111.csv"),
                                os.path.join(DATA, "xraydb_mini"), 6)
    assert pdf.shape[0] == 111
    p = Projector(g, *tabs)
    p.set_spectrum(mu, pdf, 1000.0)

    truth = phantoms.ellipsoid_phantom_torch(g.N, g.Z, g.s, g.step, seed=40, as_float=True)
    truth[:, 4:6] *= 1.1                                   # bone P and Ca +10 %
    with torch.no_grad():
        target = project(truth, p).clone()
    vol = phantoms.ellipsoid_phantom_torch(g.N, g.Z, g.s, g.step, seed=40, as_float=True)
    del truth

    # projection: per-pixel error against the FP64 oracle on 1024 rays
    with torch.no_grad():
        pred = project(vol, p)
    vol_h = vol.cpu().numpy()
    sel = [100, 460]
    sub_tabs = tuple(np.ascontiguousarray(t[sel]) for t in tabs)
    ref = O.mbfpa_forward(g.with_(V=2), sub_tabs, None, mu, pdf, 1000.0, volf=vol_h, rows=(384, 416),
                          cols=(300, 316), exact=False, want=("d",))["d"]
    got = pred[sel].cpu().numpy()
    r, c = slice(800 - 416, 800 - 384), slice(300, 316)   # rows are stored flipped (H - 1 - j)
    rel = np.abs(got[:, r, c] - ref[:, r, c]) / ref[:, r, c]
    assert rel.max() <= 1e-5, rel.max()

    # gradient: central difference of the loss along d against <grad, d>
    loss0, grad = decomposition_step(vol, target, p)
    assert abs(float(loss0) - _loss(pred, target)) <= 1e-4 * _loss(pred, target)
    _, grad_rm = decomposition_step(vol, target, p, keep_limit=0)   # path integrals re-marched
    assert float((grad_rm - grad).norm()) <= 1e-5 * float(grad.norm())
    del grad_rm
    rng = np.random.default_rng(7)
    k = 4096
    zi = torch.from_numpy(rng.integers(150, 250, k)).to(cuda)
    yi = torch.from_numpy(rng.integers(156, 356, k)).to(cuda)
    xi = torch.from_numpy(rng.integers(156, 356, k)).to(cuda)
    d = torch.zeros_like(vol)
    d[zi, 3, yi, xi] = torch.sign(grad[zi, 3, yi, xi])  # oxygen
    gd = float((grad.double() * d.double()).sum())
    h = 10.0
    with torch.no_grad():
        lp = _loss(project(vol + h * d, p), target)
        lm = _loss(project(vol - h * d, p), target)
    fd = (lp - lm) / (2 * h)
    assert gd > 0 and abs(fd - gd) <= 2e-2 * gd, (fd, gd)
    del d

    # two descent steps (backtracking on the step length) lower the loss
    loss = float(loss0)
    for _ in range(2):
        _, grad = decomposition_step(vol, target, p)
        alpha = 0.5 * loss / float((grad.double() ** 2).sum())
        for _ in range(8):
            trial = (vol - alpha * grad).clamp_(min=0.0)
            with torch.no_grad():
                lt = _loss(project(trial, p), target)
            if lt < loss:
                break
            alpha *= 0.25
        assert lt < loss
        vol, loss = trial, lt
    del grad

    # FDK of the final projections to 512x512x400 short
    with torch.no_grad():
        proj = project(vol, p).clone()
    fg = FdkGeometry(W=800, H=800, V=720, N=512, Z=400, zstart=-20, step=0.1, scale=0.05)  # z in [-20, 20) cm
    f = Fdk(fg, ang, np.zeros(fg.V), np.zeros(fg.V))
    filt = f.filter(proj, method=FILTER_BF16X3)
    proj_h = proj.cpu().numpy()
    d64 = O.filter_sinogram(proj_h[sel], np.zeros(2), np.zeros(2), O.fdk_consts(fg.piso), mode=1)
    fsel = filt[sel].cpu().numpy()
    assert np.abs(fsel - d64).max() <= 1e-5 * np.abs(d64).max()
    vf, vi = f.backproject(filt)
    filt_h = filt.cpu().numpy()
    z0 = 200                                               # slices at z = 0 and 0.1 cm
    bp64 = O.backproject(fg.N, 2, 0, fg.step, fg.scale, filt_h, fg.xfactor, ang, np.zeros(fg.V),
                         O.fdk_consts(fg.piso))
    vf2 = vf[z0:z0 + 2].cpu().numpy()
    assert np.abs(vf2 - bp64).max() <= 1e-5 * max(1.0, np.abs(bp64).max())
    vi2 = vi[z0:z0 + 2].cpu().numpy().astype(np.int32)
    assert np.abs(vi2 - np.trunc(bp64).astype(np.int32)).max() <= 1
    assert int((vi2 != 0).sum()) > 0.5 * np.pi * 256 * 256   # the body is reconstructed
