"""Error of every output against the FP64 oracle and against the reference's
own CPU code, on one seeded case each, printed as a table (run with -s to
see it) and checked against the bars: projections 1e-5 relative per pixel,
filtered projections 1e-5 of the output scale, short volume +-1 LSB,
gradient 1e-5 relative (L2)."""
import numpy as np
import pytest

import oracle as O
from tests.cases import proj_case, spectrum
from virtualcbct_b200 import FILTER_BF16X3, FILTER_DIRECT_F32, Fdk, FdkGeometry, Projector

pytestmark = pytest.mark.gpu


def _row(name, vs, err, unit, bar):
    return f"| {name} | {vs} | {err:.3e} {unit} | {bar} |"


def test_parity_report(cuda):
    import torch
    rows = ["| output | against | max error | bar |", "|---|---|---|---|"]
    # --- projection (ellipsoid phantom, 6 views incl. z_reg = 0 central row)
    g, tabs, vol, _ = proj_case("ellipsoid", seed=3, z_reg=0.0, V=6)
    mu, pdf = spectrum()
    p = Projector(g, *tabs)
    p.set_spectrum(mu, pdf, 1000.0)
    p.load_volume(vol)
    out = np.empty((g.V, g.H, g.W), np.float32)
    p.forward(out)
    ref = O.mbfpa_forward(g, tabs, vol, mu, pdf, 1000.0, exact=True, want=("f", "d"))
    e64 = float(np.max(np.abs(out - ref["d"]) / ref["d"]))
    eref = float(np.max(np.abs(out - ref["f"]) / ref["f"]))
    rows.append(_row("projection (MBFPA)", "FP64 oracle", e64, "rel/pixel", "1e-5"))
    rows.append(_row("projection (MBFPA)", "reference GPU-kernel semantics, float sum", eref, "rel/pixel", "1e-5"))
    assert e64 <= 1e-5 and eref <= 1e-5
    if O.have_reference():
        # reprojection.cpp itself (times the cos^3 factor, rows flipped); rays
        # on which its GPU and CPU twins disagree (tie rules) excluded
        cpu, _ = O.ref_mbfpa_views(g, tabs, vol, mu, pdf, 1000.0, np.arange(g.V), np.arange(pdf.shape[0]))
        leng = ref["d"] / O.mbfpa_forward(g, tabs, vol, mu, pdf, 1000.0, with_leng=False, want=("d",))["d"]
        cpu_gpu_layout = cpu[:, ::-1, :] * leng
        twin = ref["f"] != O.mbfpa_forward(g, tabs, vol, mu, pdf, 1000.0, ties=O.TIES_CPU, want=("f",))["f"]
        ecpu = float((np.abs(out - cpu_gpu_layout) / cpu_gpu_layout)[~twin].max())
        rows.append(_row("projection (MBFPA)", f"reprojection.cpp ({int(twin.sum())} tie rays excluded)", ecpu,
                         "rel/pixel", "1e-5"))
        assert ecpu <= 1e-5
    # --- FDK
    rng = np.random.default_rng(0)
    V, H, W = 12, 40, 48
    base = rng.uniform(0.05, 1.0, size=(V, H, W)).astype(np.float32)
    k = np.ones(5) / 5
    for ax in (1, 2):
        base = np.apply_along_axis(lambda r: np.convolve(r, k, mode="same"), ax, base)
    proj = np.clip(base, 0.02, 1.0).astype(np.float32)
    ang = np.deg2rad(-180.0001 + np.arange(V) * 360.0 / V)
    fg = FdkGeometry(W=W, H=H, V=V, N=27, Z=8, zstart=-3, step=0.5, scale=0.4)
    xs = np.full(V, 2.0)
    f = Fdk(fg, ang, xs, np.zeros(V))
    d64 = O.filter_sinogram(proj, xs, np.zeros(V), O.fdk_consts(fg.piso), mode=1)
    scale = np.abs(d64).max()
    for method, name in ((FILTER_DIRECT_F32, "direct FP32"), (FILTER_BF16X3, "tcgen05 BF16x3")):
        filt = f.filter(proj, method=method)
        e = float(np.abs(filt - d64).max() / scale)
        rows.append(_row(f"filtered projections ({name})", "FP64 filter", e, "of output scale", "1e-5"))
        assert e <= 1e-5
    filt = f.filter(proj, method=FILTER_DIRECT_F32)
    vf, vi = f.backproject(filt)
    bp64 = O.backproject(fg.N, fg.Z, fg.zstart, fg.step, fg.scale, filt, fg.xfactor, ang, xs,
                         O.fdk_consts(fg.piso))
    ebp = float(np.abs(vf - bp64).max() / max(1.0, np.abs(bp64).max()))
    rows.append(_row("volume before the cast (BP)", "FP64 backprojection of the same filter", ebp, "of volume scale",
                     "1e-5"))
    assert ebp <= 1e-5
    if O.have_reference():
        rfilt, _ = O.ref_filter(proj, xs, np.zeros(V), fg.piso)
        rvol, _ = O.ref_backproject(fg.N, fg.Z, fg.zstart, fg.step, fg.scale, rfilt, fg.xfactor, ang, xs, fg.piso)
        _, vi2 = f.reconstruct(proj)
        lsb = int(np.abs(vi2.astype(np.int32) - rvol.astype(np.int16).astype(np.int32)).max())
        rows.append(f"| short volume (filter + BP + cast) | filterSinogram + reconstructImage | {lsb} LSB | 1 LSB |")
        assert lsb <= 1
    # --- adjoint
    g2, tabs2, vol2, _ = proj_case("ellipsoid", seed=0)
    volf = vol2.astype(np.float32) * np.random.default_rng(0).uniform(0.9, 1.1, size=vol2.shape).astype(np.float32)
    resid = np.random.default_rng(100).normal(size=(g2.V, g2.H, g2.W)).astype(np.float32)
    p2 = Projector(g2, *tabs2)
    p2.set_spectrum(mu, pdf, 1000.0)
    p2.load_volume_f32(torch.from_numpy(volf).to(cuda))
    gpu = p2.adjoint(torch.from_numpy(resid).to(cuda)).cpu().numpy().astype(np.float64)
    gref = O.mbfpa_adjoint(g2, tabs2, volf, mu, pdf, 1000.0, resid.astype(np.float64))
    eg = float(np.linalg.norm(gpu - gref) / np.linalg.norm(gref))
    rows.append(_row("gradient (adjoint)", "FP64 oracle gradient", eg, "rel (L2)", "1e-5"))
    assert eg <= 1e-5
    print("\n" + "\n".join(rows))
