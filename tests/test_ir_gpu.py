"""Iterative-reconstruction helpers on the GPU against the oracle
restatement (itself bitwise the reference's lengthproj / IR_ImageCBCT):
bitwise, since the kernels follow the same double arithmetic without FMA
contraction."""
import numpy as np
import pytest

import oracle as O
from tests.test_ir_cpu import ir_case
from virtualcbct_b200 import Projector, _native
from virtualcbct_b200.iterative import ir_update

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ite,xshift,views", [(0, 0.0, None), (1, 1.2, (1, 4)), (0, -0.7, (0, 5))])
def test_lengthproj_matches_oracle(cuda, ite, xshift, views):
    import torch
    g, tabs, proj = ir_case(seed=ite + 3, xshift=xshift)
    p = Projector(g, *tabs)
    ref = O.lengthproj(g, tabs, proj, ite=ite, views=views)
    host = p.lengthproj(proj, ite=ite, views=views)
    dev = p.lengthproj(torch.from_numpy(proj.view(np.int16)).to(cuda), ite=ite, views=views).cpu().numpy()
    assert np.array_equal(host, ref), np.abs(host - ref).max()
    assert np.array_equal(dev, ref)


def test_lengthproj_reference_named_entry_point(cuda):
    import ctypes as C
    g, tabs, proj = ir_case(seed=9)
    ref = O.lengthproj(g, tabs, proj, ite=0)
    npf = np.zeros((g.Z, g.N, g.N), np.float32)
    cosT, sinT, Xc, Yc = [np.ascontiguousarray(t, np.float64) for t in tabs]
    dp = C.POINTER(C.c_double)
    L = _native.lib()
    L.vcbct_lengthproj(0, g.N, g.Z, None, None, npf.ctypes.data_as(C.POINTER(C.c_float)), C.c_void_p(proj.ctypes.data),
                 g.s, g.step, g.W, g.H, 0, g.V, None, cosT.ctypes.data_as(dp), sinT.ctypes.data_as(dp),
                 Xc.ctypes.data_as(dp), Yc.ctypes.data_as(dp), 0.0, None, g.pdet, g.piso, g.sad, g.dpn,
                 g.x_reg, g.y_reg, g.z_reg)
    assert np.array_equal(npf, ref)


@pytest.mark.parametrize("wtv", [0.0, 0.002])
def test_ir_update_matches_oracle(cuda, wtv):
    import torch
    rng = np.random.default_rng(11)
    N, Z = 40, 9
    before = rng.integers(0, 3000, size=(Z, N, N)).astype(np.int16)
    npf = rng.uniform(1.0, 5.0, size=(Z, N, N)).astype(np.float32)
    npf_re = rng.uniform(1.0, 5.0, size=(Z, N, N)).astype(np.float32)
    ref = O.ir_update(N, Z, 0.1, before, npf, npf_re, 0.3, wtv, 0.0)
    host = ir_update(before, npf, npf_re, 0.1, 0.3, wtv)
    dev = ir_update(*(torch.from_numpy(a).to(cuda) for a in (before, npf, npf_re)), 0.1, 0.3, wtv).cpu().numpy()
    assert np.array_equal(host, ref)
    assert np.array_equal(dev, ref)
