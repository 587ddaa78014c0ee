"""MBFPA parity: the CUDA projector (through the C ABI) against the FP64
oracle restatement of reprojectionKernel and against the reference's own CPU
projector (oracle/_ref), on seeded inputs."""
import numpy as np
import pytest

import oracle as O
from tests.cases import proj_case, spectrum
from virtualcbct_b200 import Projector

pytestmark = pytest.mark.gpu

# Parity bar for projections: 1e-5 relative per detector pixel.
RTOL = 1e-5


def _gpu_forward(g, tabs, vol, mu, pdf, xf=1000.0):
    p = Projector(g, *tabs)
    p.set_spectrum(mu, pdf, xf)
    p.load_volume(vol)
    out = np.empty((g.V, g.H, g.W), np.float32)
    p.forward(out)
    return out, p


CASES = [
    ("random", 0, {}),
    ("random", 1, {}),
    ("water", 0, {}),
    ("ellipsoid", 3, {}),
    # half-fan detector offset (projector xshift x100 px)
    ("random", 2, dict(xshift=1.6, W=40, H=32)),
    # thin slices: several z crossings per x step on some rays
    ("ellipsoid", 5, dict(N=48, Z=40, s=0.25, step=0.1, V=3)),
    # voxel size whose reciprocal is not an integer: dominant-axis planes fall
    # inside the steps
    ("random", 9, dict(N=40, Z=24, s=0.07, step=0.13, V=3)),
    # steeper than one slice per step: the per-step march path
    ("random", 6, dict(N=32, Z=64, s=0.3, step=0.02, V=2, W=24, H=40, dpn=900.0)),
    # z_reg = 0: the central detector row lies exactly in the z = 0 plane, a
    # slice boundary (the reference's (int)(nzm - z/step) rule applies)
    ("ellipsoid", 7, dict(z_reg=0.0, V=6)),
    ("random", 8, dict(z_reg=0.0, N=32, Z=64, s=0.3, step=0.02, V=2, W=24, H=40, dpn=900.0)),
    # one view of a 5 x 3 detector: a warp with 3 of 32 rows, a partial block
    # of columns
    ("ellipsoid", 11, dict(V=1, W=5, H=3)),
]


@pytest.mark.parametrize("kind,seed,extra", CASES)
def test_forward_matches_fp64_oracle(cuda, kind, seed, extra):
    g, tabs, vol, _ = proj_case(kind, seed=seed, **extra)
    mu, pdf = spectrum()
    gpu, _ = _gpu_forward(g, tabs, vol, mu, pdf)
    ref = O.mbfpa_forward(g, tabs, vol, mu, pdf, 1000.0, exact=True, want=("f", "d"))
    rel = np.abs(gpu.astype(np.float64) - ref["d"]) / ref["d"]
    assert np.isfinite(gpu).all()
    assert rel.max() <= RTOL, f"max rel err {rel.max():.3e} at {np.unravel_index(rel.argmax(), rel.shape)}"


def test_forward_matches_reference_cpu_twin(cuda):
    """Against reprojection.cpp itself (times the cos^3 factor, rows flipped);
    rays on which the reference's GPU and CPU twins disagree (tie rules) are
    compared with the GPU-semantics oracle instead."""
    if not O.have_reference():
        pytest.skip("reference CPU objects not built")
    g, tabs, vol, _ = proj_case("random", seed=2)
    mu, pdf = spectrum()
    gpu, _ = _gpu_forward(g, tabs, vol, mu, pdf)
    bins = np.arange(pdf.shape[0])
    cpu, _ = O.ref_mbfpa_views(g, tabs, vol, mu, pdf, 1000.0, np.arange(g.V), bins)
    og = O.mbfpa_forward(g, tabs, vol, mu, pdf, 1000.0, ties=O.TIES_GPU, want=("f", "d"))
    oc = O.mbfpa_forward(g, tabs, vol, mu, pdf, 1000.0, ties=O.TIES_CPU, with_leng=False, flip=False, want=("f",))
    assert np.array_equal(oc["f"], cpu)  # the oracle is pinned to the reference
    leng = og["d"] / O.mbfpa_forward(g, tabs, vol, mu, pdf, 1000.0, with_leng=False, want=("d",))["d"]
    cpu_gpu_layout = cpu[:, ::-1, :] * leng
    twin = og["f"] != O.mbfpa_forward(g, tabs, vol, mu, pdf, 1000.0, ties=O.TIES_CPU, want=("f",))["f"]
    rel = np.abs(gpu - cpu_gpu_layout) / cpu_gpu_layout
    assert rel[~twin].max() <= RTOL
    rel_t = np.abs(gpu.astype(np.float64) - og["d"]) / og["d"]
    assert rel_t[twin].max(initial=0.0) <= RTOL


def test_segment_count_matches_oracle(cuda):
    g, tabs, vol, _ = proj_case("water")
    mu, pdf = spectrum()
    _, p = _gpu_forward(g, tabs, vol, mu, pdf)
    ref = O.mbfpa_forward(g, tabs, vol, mu, pdf, 1000.0, exact=False, want=("nm",))
    n_gpu = p.count_segments()
    n_ref = int(ref["nm"].sum())
    assert abs(n_gpu - n_ref) <= 1e-4 * n_ref


def test_path_integrals_match_oracle(cuda):
    g, tabs, vol, _ = proj_case("random", seed=5)
    mu, pdf = spectrum()
    _, p = _gpu_forward(g, tabs, vol, mu, pdf)
    L = p.path_integrals().cpu().numpy()
    ref = O.mbfpa_forward(g, tabs, vol, mu, pdf, 1000.0, exact=False, want=("L",))["L"]
    scale = np.abs(ref).max()
    assert np.abs(L - ref).max() <= 2e-5 * scale
