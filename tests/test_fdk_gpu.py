"""FDK parity: the CUDA filter and backprojector (through the C ABI) against
the reference's own filterSinogram / reconstructImage (oracle/_ref) and the
FP64 oracle restatement, on seeded projections."""
import numpy as np
import pytest

import oracle as O
from virtualcbct_b200 import FILTER_BF16X3, FILTER_DIRECT_F32, Fdk, FdkGeometry, redundancy_weights

pytestmark = pytest.mark.gpu


def _case(V=6, H=40, W=48, seed=0, N=27, Z=8, span=360.0, xshift=0.0):
    rng = np.random.default_rng(seed)
    # smooth positive "projections" in (0, 1]: a blurred random field
    base = rng.uniform(0.05, 1.0, size=(V, H, W)).astype(np.float32)
    k = np.ones(5) / 5
    for ax in (1, 2):
        base = np.apply_along_axis(lambda r: np.convolve(r, k, mode="same"), ax, base)
    proj = np.clip(base, 0.02, 1.0).astype(np.float32)
    ang = np.deg2rad(-180.0001 + np.arange(V) * span / V)
    g = FdkGeometry(W=W, H=H, V=V, N=N, Z=Z, zstart=-3, step=0.5, scale=0.4)
    xs = np.full(V, xshift)
    return g, proj, ang, xs


def test_filter_matches_reference(cuda):
    if not O.have_reference():
        pytest.skip("reference CPU objects not built")
    g, proj, ang, xs = _case()
    f = Fdk(g, ang, xs, np.zeros(g.V))
    gpu = f.filter(proj, method=FILTER_DIRECT_F32)
    ref, _ = O.ref_filter(proj, xs, np.zeros(g.V), g.piso)
    d64 = O.filter_sinogram(proj, xs, np.zeros(g.V), O.fdk_consts(g.piso), mode=1)
    scale = np.abs(d64).max()
    # the reference itself accumulates in float; both sit within 1e-5 of the
    # output scale of the FP64 filter
    assert np.abs(ref - d64).max() <= 1e-5 * scale
    assert np.abs(gpu - d64).max() <= 1e-5 * scale


def test_filter_with_offset_detector(cuda):
    g, proj, ang, xs = _case(xshift=3.0)
    f = Fdk(g, ang, xs, np.zeros(g.V))
    gpu = f.filter(proj)
    d64 = O.filter_sinogram(proj, xs, np.zeros(g.V), O.fdk_consts(g.piso), mode=1)
    assert np.abs(gpu - d64).max() <= 1e-5 * np.abs(d64).max()


@pytest.mark.parametrize("method", [FILTER_DIRECT_F32, FILTER_BF16X3])
def test_redundancy_weighted_filter_matches_fp64(cuda, method):
    """With redundancy = 1 both filters weight -log p by the half-fan
    redundancy weights before filtering: against the FP64 filter of
    w * (-log p), given as p ** w."""
    g, proj, ang, xs = _case(xshift=3.0)
    g = g.with_(redundancy=1)
    w = redundancy_weights(g, xs)
    assert w.min() == 0.0 and w.max() == 2.0
    f = Fdk(g, ang, xs, np.zeros(g.V))
    gpu = f.filter(proj, method=method)
    pw = (proj.astype(np.float64) ** w[:, None, :].astype(np.float64)).astype(np.float32)
    d64 = O.filter_sinogram(pw, xs, np.zeros(g.V), O.fdk_consts(g.piso), mode=1)
    assert np.abs(gpu - d64).max() <= 1e-5 * np.abs(d64).max()


@pytest.mark.parametrize("xshift", [0.0, 2.0])
def test_backprojection_matches_reference(cuda, xshift):
    if not O.have_reference():
        pytest.skip("reference CPU objects not built")
    g, proj, ang, xs = _case(V=12, xshift=xshift)
    filt, _ = O.ref_filter(proj, xs, np.zeros(g.V), g.piso)
    f = Fdk(g, ang, xs, np.zeros(g.V))
    vf, vi = f.backproject(filt)
    ref, _ = O.ref_backproject(g.N, g.Z, g.zstart, g.step, g.scale, filt, g.xfactor, ang, xs, g.piso)
    ref_i16 = ref.astype(np.int16)  # (short) truncation toward zero (R/main.cpp:184)
    assert np.abs(vf - ref).max() <= 1e-5 * max(1.0, np.abs(ref).max())
    assert np.abs(vi.astype(np.int32) - ref_i16.astype(np.int32)).max() <= 1


def test_odd_sizes_match_reference(cuda):
    """Odd detector and volume sizes (H / 2 and W / 2 round down as in the
    reference; a partial slice block; warps cut by the volume's edge) and an
    offset detector: filter against the FP64 filter, backprojection and short
    volume against reconstructImage."""
    if not O.have_reference():
        pytest.skip("reference CPU objects not built")
    g, proj, ang, xs = _case(V=7, H=41, W=47, N=33, Z=11, seed=5, xshift=1.0)
    f = Fdk(g, ang, xs, np.zeros(g.V))
    gpu = f.filter(proj, method=FILTER_DIRECT_F32)
    d64 = O.filter_sinogram(proj, xs, np.zeros(g.V), O.fdk_consts(g.piso), mode=1)
    assert np.abs(gpu - d64).max() <= 1e-5 * np.abs(d64).max()
    filt, _ = O.ref_filter(proj, xs, np.zeros(g.V), g.piso)
    vf, vi = f.backproject(filt)
    ref, _ = O.ref_backproject(g.N, g.Z, g.zstart, g.step, g.scale, filt, g.xfactor, ang, xs, g.piso)
    assert np.abs(vf - ref).max() <= 1e-5 * max(1.0, np.abs(ref).max())
    assert np.abs(vi.astype(np.int32) - ref.astype(np.int16).astype(np.int32)).max() <= 1


def test_fdk_chain_short_volume_within_one_lsb(cuda):
    if not O.have_reference():
        pytest.skip("reference CPU objects not built")
    g, proj, ang, xs = _case(V=24, H=48, W=64, N=40, Z=10, seed=3)
    f = Fdk(g, ang, xs, np.zeros(g.V))
    _, vi = f.reconstruct(proj)
    filt, _ = O.ref_filter(proj, xs, np.zeros(g.V), g.piso)
    ref, _ = O.ref_backproject(g.N, g.Z, g.zstart, g.step, g.scale, filt, g.xfactor, ang, xs, g.piso)
    d = np.abs(vi.astype(np.int32) - ref.astype(np.int16).astype(np.int32))
    assert d.max() <= 1, f"{(d > 1).sum()} voxels differ by more than 1 LSB"


@pytest.mark.parametrize("V,H,W,xshift", [(6, 40, 48, 0.0), (4, 8, 400, 0.0), (3, 100, 400, 16.0),
                                          (2, 70, 256, 2.0), (3, 10, 50, 0.0), (3, 20, 47, 1.0),
                                          # wider than one 512-column accumulator: column tiles
                                          (2, 12, 600, 0.0), (2, 9, 800, 8.0), (2, 5, 1030, 0.0)])
def test_bf16x3_tensor_core_filter_matches_fp64(cuda, V, H, W, xshift):
    """The tcgen05 BF16 3-term split GEMM against the FP64 filter; the same
    tolerance as the direct FP32 path (1e-5 of the output scale) up to 800
    columns (the widest detector of the workloads).  The tensor cores' FP32
    accumulation error grows with the number of K steps; at 1030 columns it
    reaches about 1.1e-5 of the scale, so that width is held to 3e-5 (it
    checks the three column tiles)."""
    from virtualcbct_b200 import FILTER_BF16X3
    tol = 1e-5 if W <= 800 else 3e-5
    g, proj, ang, xs = _case(V=V, H=H, W=W, seed=W + V, xshift=xshift)
    f = Fdk(g, ang, xs, np.zeros(g.V))
    gpu = f.filter(proj, method=FILTER_BF16X3)
    d64 = O.filter_sinogram(proj, xs, np.zeros(g.V), O.fdk_consts(g.piso), mode=1)
    assert np.isfinite(gpu).all()
    assert np.abs(gpu - d64).max() <= tol * np.abs(d64).max()
    direct = f.filter(proj, method=FILTER_DIRECT_F32)
    assert np.abs(direct - d64).max() <= 1e-5 * np.abs(d64).max()
    assert np.abs(gpu - direct).max() <= tol * np.abs(d64).max()


@pytest.mark.parametrize("redundancy", [0, 1])
def test_bf16x3_fused_and_split_a_operand_agree(cuda, redundancy):
    """Device projections with 16-byte-aligned rows take the fused form (the
    GEMM makes the A planes of -ln p in shared memory); the same values at a
    4-byte offset take the split pass through global memory.  Both against
    the FP64 filter at 1e-5 of the scale, with and without redundancy
    weights."""
    import torch
    g, proj, ang, xs = _case(V=3, H=70, W=400, seed=11, xshift=2.0)
    g = g.with_(redundancy=redundancy)
    f = Fdk(g, ang, xs, np.zeros(g.V))
    if redundancy:
        w = redundancy_weights(g, xs)
        pw = (proj.astype(np.float64) ** w[:, None, :].astype(np.float64)).astype(np.float32)
    else:
        pw = proj
    d64 = O.filter_sinogram(pw, xs, np.zeros(g.V), O.fdk_consts(g.piso), mode=1)
    n = proj.size
    aligned = torch.from_numpy(proj).cuda()
    store = torch.empty(n + 1, dtype=torch.float32, device="cuda")
    offset = store[1:].view(proj.shape)
    offset.copy_(aligned)
    assert aligned.data_ptr() % 16 == 0 and offset.data_ptr() % 16 == 4
    fused = f.filter(aligned, method=FILTER_BF16X3).cpu().numpy()
    split = f.filter(offset, method=FILTER_BF16X3).cpu().numpy()
    scale = np.abs(d64).max()
    assert np.abs(fused - d64).max() <= 1e-5 * scale
    assert np.abs(split - d64).max() <= 1e-5 * scale
    assert np.abs(fused - split).max() <= 1e-5 * scale


def test_bf16x3_unaligned_output_and_short_views(cuda):
    """An output 4 bytes off alignment takes the unfused form (the fused one
    stores through TMA); views of fewer than 8 rows take the per-row weight
    loads of the fused converter.  Both against the FP64 filter of
    w * (-log p) at 1e-5 of the scale."""
    import torch
    g, proj, ang, xs = _case(V=5, H=5, W=64, seed=21, xshift=3.0)
    g = g.with_(redundancy=1)
    w = redundancy_weights(g, xs)
    f = Fdk(g, ang, xs, np.zeros(g.V))
    pw = (proj.astype(np.float64) ** w[:, None, :].astype(np.float64)).astype(np.float32)
    d64 = O.filter_sinogram(pw, xs, np.zeros(g.V), O.fdk_consts(g.piso), mode=1)
    scale = np.abs(d64).max()
    p = torch.from_numpy(proj).cuda()
    fused = f.filter(p, method=FILTER_BF16X3).cpu().numpy()
    store = torch.empty(proj.size + 1, dtype=torch.float32, device="cuda")
    out = store[1:].view(proj.shape)
    assert out.data_ptr() % 16 == 4
    f.filter(p, out, method=FILTER_BF16X3)
    split = out.cpu().numpy()
    assert np.abs(fused - d64).max() <= 1e-5 * scale
    assert np.abs(split - d64).max() <= 1e-5 * scale
