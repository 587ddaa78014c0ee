"""The scratch-free forward projection (vcbct_mbfpa_forward_noalloc).

It exists for callers that cannot let a library allocate device memory (hosts
that own all memory in a fixed arena, latency-critical pipelines, deployments
that forbid allocation after start-up).  These tests call it through the C ABI
and check it on two calls in a row, with different volumes and sizes (so that
anything left in its shared scratch array by the first call would show in the
second), against the FP64 oracle (the independent check) and against the
object API's forward projection.  The host tables handed to each call are
overwritten as soon as it returns: the entry point copies them before
returning.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from tests.cases import proj_case, spectrum
from virtualcbct_b200 import Projector, _native as N

RTOL = 1e-5  # the projector parity tolerance used throughout the tests


def _dp(a):
    return np.ascontiguousarray(a, np.float64).ctypes.data_as(C.POINTER(C.c_double))


def _noalloc(g, tabs, vol_dev, mu, pdf, out_dev, stream):
    tabs = [np.array(t, np.float64) for t in tabs]
    mu = np.array(mu, np.float32)
    pdf = np.array(pdf, np.float32)
    gc = g.to_c()
    rc = N.lib().vcbct_mbfpa_forward_noalloc(
        C.byref(gc), *[t.ctypes.data_as(C.POINTER(C.c_double)) for t in tabs],
        C.c_void_p(vol_dev.data_ptr()), mu.ctypes.data_as(C.POINTER(C.c_float)),
        pdf.ctypes.data_as(C.POINTER(C.c_float)), int(pdf.shape[0]), 1000.0,
        C.c_void_p(out_dev.data_ptr()), C.c_void_p(stream.cuda_stream))
    # the call has copied its host inputs: spoil them before the GPU runs
    for a in (*tabs, mu, pdf):
        a.fill(np.nan)
    return rc


@pytest.mark.gpu
def test_noalloc_forward_matches_object_api_on_two_calls(cuda):
    import torch
    stream = torch.cuda.current_stream()
    mu, pdf = spectrum()
    cases = [proj_case("random", N=64, Z=16, seed=7, hi=400),
             proj_case("ellipsoid", N=48, Z=12, W=40, H=36, V=3, seed=2)]
    for g, tabs, vol, _ in cases:
        vd = torch.from_numpy(vol.view(np.int16)).to(cuda)
        out = torch.full((g.V, g.H, g.W), float("nan"), device=cuda)
        rc = _noalloc(g, tabs, vd, mu, pdf, out, stream)
        assert rc == 0, N.lib().vcbct_last_error()
        p = Projector(g, *tabs)
        p.set_spectrum(mu, pdf, 1000.0)
        p.load_volume(vd)
        ref = p.forward()
        torch.cuda.synchronize()
        a, b = out.cpu().numpy(), ref.cpu().numpy()
        assert np.isfinite(a).all()
        assert np.max(np.abs(a - b) / b) <= RTOL
        d64 = O.mbfpa_forward(g, tabs, vol, mu, pdf, 1000.0, exact=False, want=("d",))["d"]
        assert np.max(np.abs(a - d64) / d64) <= RTOL


def test_noalloc_rejects_sizes_beyond_its_scratch():
    from virtualcbct_b200 import ProjGeometry
    g = ProjGeometry(N=512, Z=100, s=0.05, step=0.2, W=8, H=8, V=2)
    t = np.zeros(2)
    gc = g.to_c()
    rc = N.lib().vcbct_mbfpa_forward_noalloc(C.byref(gc), _dp(t), _dp(t), _dp(t), _dp(t),
                                             C.c_void_p(1), np.zeros(6, np.float32).ctypes.data_as(C.POINTER(C.c_float)),
                                             np.zeros(1, np.float32).ctypes.data_as(C.POINTER(C.c_float)),
                                             1, 1000.0, C.c_void_p(1), None)
    assert rc == 3
    assert b"4177920" in N.lib().vcbct_last_error()
