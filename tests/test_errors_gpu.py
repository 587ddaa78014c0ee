"""State errors of live objects: a projector used before it has a volume or
a spectrum, the adjoint before a volume, a batch given a projector without a
volume, an unknown filter method, an invalid view range -- each a status and
a message, with the object still usable afterwards."""
import ctypes as C

import numpy as np
import pytest

from tests.cases import proj_case, spectrum
from virtualcbct_b200 import Batch, Fdk, FdkGeometry, Projector
from virtualcbct_b200 import _native as N

pytestmark = pytest.mark.gpu

ARG, LIMIT, STATE = 1, 3, 4


def _rc(fn, *args):
    rc = fn(*args)
    return rc, N.lib().vcbct_last_error().decode()


def test_projector_state_errors(cuda):
    import torch
    L = N.lib()
    g, tabs, vol, _ = proj_case("random", seed=0)
    p = Projector(g, *tabs)
    out = torch.empty((g.V, g.H, g.W), dtype=torch.float32, device=cuda)
    rc, msg = _rc(L.vcbct_projector_forward, p._h, C.c_void_p(out.data_ptr()), 1, None)
    assert rc == STATE and "volume" in msg
    grad = torch.zeros((g.Z, g.nmat, g.N, g.N), dtype=torch.float32, device=cuda)
    rc, msg = _rc(L.vcbct_projector_adjoint, p._h, C.c_void_p(out.data_ptr()), C.c_void_p(grad.data_ptr()), None)
    assert rc == STATE and "volume" in msg
    p.load_volume(vol)
    rc, msg = _rc(L.vcbct_projector_forward, p._h, C.c_void_p(out.data_ptr()), 1, None)
    assert rc == STATE and "spectrum" in msg
    mu, pdf = spectrum()
    big = np.zeros(2000, np.float32)
    rc, msg = _rc(L.vcbct_projector_set_spectrum, p._h, big.ctypes.data_as(C.POINTER(C.c_float)),
                  big.ctypes.data_as(C.POINTER(C.c_float)), 2000, 1000.0)
    assert rc == LIMIT
    p.set_spectrum(mu, pdf, 1000.0)
    rc, _ = _rc(L.vcbct_projector_set_noise, p._h, 3, 1e4, 6e4, 0)
    assert rc == ARG
    proj = np.zeros((g.V, g.H, g.W), np.uint16)
    npf = np.zeros((g.Z, g.N, g.N), np.float32)
    rc, _ = _rc(L.vcbct_projector_lengthproj, p._h, 0, 2, 1, C.c_void_p(proj.ctypes.data), 0,
                C.c_void_p(npf.ctypes.data), 0, None)
    assert rc == ARG
    p.forward(out)                              # still usable
    assert torch.isfinite(out).all()


def test_batch_and_fdk_state_errors(cuda):
    import torch
    g, tabs, vol, _ = proj_case("random", seed=1)
    mu, pdf = spectrum()
    p = Projector(g, *tabs)
    p.set_spectrum(mu, pdf, 1000.0)
    b = Batch()
    out = torch.empty((g.V, g.H, g.W), dtype=torch.float32, device=cuda)
    with pytest.raises(N.VcbctError, match="volume"):
        b.add(p, out)
    fg = FdkGeometry(W=48, H=40, V=6, N=27, Z=8, zstart=-3, step=0.5, scale=0.4)
    ang = np.deg2rad(-180.0001 + np.arange(6) * 60.0)
    f = Fdk(fg, ang, np.zeros(6), np.zeros(6))
    proj = np.full((6, 40, 48), 0.5, np.float32)
    with pytest.raises(N.VcbctError, match="method"):
        f.filter(proj, method=7)
    assert np.isfinite(f.filter(proj)).all()    # still usable
