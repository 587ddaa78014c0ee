"""Argument validation of the C ABI, on the CPU: every entry point given NULL
handles or buffers, out-of-range sizes or unreadable files returns a status
(VCBCT_ERR_ARG 1, _LIMIT 3, _STATE 4, _IO 5) with a message, without a CUDA
call -- the reference prints and exits instead (reprojectionOnGPU.cu:846-880,
filterSinogram.cpp NULL checks)."""
import ctypes as C

import numpy as np
import pytest

from virtualcbct_b200 import _native as N
from virtualcbct_b200 import FdkGeometry, ProjGeometry

ARG, LIMIT, STATE, IO = 1, 3, 4, 5


@pytest.fixture(scope="module")
def L():
    return N.lib()


def _msg(L):
    return L.vcbct_last_error().decode()


def test_null_projector_handles(L):
    f = np.zeros(4, np.float32)
    fp = f.ctypes.data_as(C.POINTER(C.c_float))
    assert L.vcbct_projector_destroy(None) == 0
    assert L.vcbct_projector_set_spectrum(None, fp, fp, 2, 1000.0) == ARG
    assert L.vcbct_projector_load_volume(None, None, 0, None) == ARG
    assert L.vcbct_projector_load_volume_f32(None, None, 1, None) == ARG
    assert L.vcbct_projector_forward(None, None, 0, None) == ARG
    assert L.vcbct_projector_project(None, None, None, None) == ARG
    assert L.vcbct_projector_set_noise(None, 1, 1e4, 6e4, 0) == ARG
    assert L.vcbct_projector_path_integrals(None, None, None) == ARG
    tot = C.c_ulonglong()
    assert L.vcbct_projector_count_segments(None, C.byref(tot), None) == ARG
    assert L.vcbct_projector_adjoint(None, None, None, None) == ARG
    assert L.vcbct_projector_forward_state(None, None, None, None) == ARG
    assert L.vcbct_projector_adjoint_state(None, None, None, None, None) == ARG
    assert L.vcbct_projector_autotune(None, None, None, None) == ARG
    assert L.vcbct_projector_lengthproj(None, 0, 0, 1, None, 0, None, 1, None) == ARG
    assert L.vcbct_projector_load_deck(None, None, None, None) == ARG
    assert "NULL" in _msg(L)


def test_null_batch_and_fdk_handles(L):
    assert L.vcbct_batch_create(None) == ARG
    assert L.vcbct_batch_destroy(None) == 0
    assert L.vcbct_batch_add(None, None, None) == ARG
    assert L.vcbct_batch_forward(None, 1, None) == ARG
    assert L.vcbct_batch_configure(None, 0, 4) == ARG
    c = C.c_int()
    assert L.vcbct_batch_autotune(None, None, C.byref(c)) == ARG
    assert L.vcbct_fdk_destroy(None) == 0
    assert L.vcbct_fdk_set_kernel(None, None) == ARG
    assert L.vcbct_fdk_filter(None, None, None, 0, 0, None) == ARG
    assert L.vcbct_fdk_backproject(None, None, None, None, 0, None) == ARG


def test_fdk_create_rejects_bad_geometry(L):
    a = np.zeros(4)
    dp = a.ctypes.data_as(C.POINTER(C.c_double))
    h = C.c_void_p()
    g = FdkGeometry(W=8, H=8, V=1, N=4, Z=2).to_c()           # one view: no angular step
    assert L.vcbct_fdk_create(C.byref(g), dp, dp, dp, C.byref(h)) == ARG and h.value is None
    g = FdkGeometry(W=8, H=8, V=4, N=4, Z=2, piso=0.0).to_c()
    assert L.vcbct_fdk_create(C.byref(g), dp, dp, dp, C.byref(h)) == ARG
    assert "positive" in _msg(L)
    g = FdkGeometry(W=8, H=8, V=4, N=4, Z=2).to_c()
    assert L.vcbct_fdk_create(C.byref(g), None, dp, dp, C.byref(h)) == ARG


def test_projector_limits(L):
    t = np.zeros(4)
    dp = t.ctypes.data_as(C.POINTER(C.c_double))
    h = C.c_void_p()
    g = ProjGeometry(N=2048, Z=1024, s=0.1, step=0.1, W=8, H=8, V=4).to_c()   # 4.3e9 voxels
    assert L.vcbct_projector_create(C.byref(g), dp, dp, dp, dp, C.byref(h)) == LIMIT
    g = ProjGeometry(N=8, Z=4, s=0.1, step=-0.1, W=8, H=8, V=4).to_c()
    assert L.vcbct_projector_create(C.byref(g), dp, dp, dp, dp, C.byref(h)) == ARG
    g = ProjGeometry(N=8, Z=4, s=0.1, step=0.1, W=8, H=8, V=4).to_c()
    assert L.vcbct_projector_create(C.byref(g), None, dp, dp, dp, C.byref(h)) == ARG


def test_noalloc_limits_before_any_device_call(L):
    t = np.zeros(2048)
    dp = t.ctypes.data_as(C.POINTER(C.c_double))
    f = np.zeros(8, np.float32)
    fp = f.ctypes.data_as(C.POINTER(C.c_float))
    buf = C.c_void_p(16)   # never dereferenced: the call fails on its limits first
    g = ProjGeometry(N=8, Z=4, s=0.1, step=0.1, W=8, H=8, V=2000).to_c()
    assert L.vcbct_mbfpa_forward_noalloc(C.byref(g), dp, dp, dp, dp, buf, fp, fp, 1, 1000.0, buf, None) == LIMIT
    g = ProjGeometry(N=2048, Z=64, s=0.1, step=0.1, W=8, H=8, V=2).to_c()
    assert L.vcbct_mbfpa_forward_noalloc(C.byref(g), dp, dp, dp, dp, buf, fp, fp, 1, 1000.0, buf, None) == LIMIT
    g = ProjGeometry(N=8, Z=4, s=0.1, step=0.1, W=8, H=8, V=2).to_c()
    assert L.vcbct_mbfpa_forward_noalloc(C.byref(g), dp, dp, dp, dp, buf, fp, fp, 2000, 1000.0, buf, None) == ARG
    assert L.vcbct_mbfpa_forward_noalloc(C.byref(g), dp, dp, dp, dp, None, fp, fp, 1, 1000.0, buf, None) == ARG
    # non-finite xfactor or geometry: rejected, as vcbct_projector_set_spectrum / _create do
    for xf in (float("inf"), float("-inf"), float("nan")):
        assert L.vcbct_mbfpa_forward_noalloc(C.byref(g), dp, dp, dp, dp, buf, fp, fp, 1, xf, buf, None) == ARG
    for field in ("z_reg", "x_reg", "recon_scale", "sad_cm"):
        g = ProjGeometry(N=8, Z=4, s=0.1, step=0.1, W=8, H=8, V=2).to_c()
        setattr(g, field, float("inf") if field in ("recon_scale", "sad_cm") else float("nan"))
        assert L.vcbct_mbfpa_forward_noalloc(C.byref(g), dp, dp, dp, dp, buf, fp, fp, 1, 1000.0, buf, None) == ARG
        assert "finite" in _msg(L) or "positive" in _msg(L)


def test_standalone_kernels_validate_arguments(L):
    assert L.vcbct_gaussian_noise(None, 4, 65535.0, 0, 1, None) == ARG
    assert L.vcbct_ir_update(4, 4, 0.1, None, None, None, None, 0.5, 0.0, 0.0, 0, None) == ARG
    s = np.zeros(16, np.int16)
    f = np.zeros(16, np.float32)
    sp, fp = C.c_void_p(s.ctypes.data), C.c_void_p(f.ctypes.data)
    assert L.vcbct_ir_update(0, 4, 0.1, sp, fp, fp, fp, 0.5, 0.0, 0.0, 0, None) == ARG
    t = N.PhantomTablesC()
    assert L.vcbct_organs_to_elements(None, 4, 1, C.byref(t), None, 0, None) == ARG
    ids = np.zeros(4, np.uint8)
    out = np.zeros(24, np.uint16)
    ip, op = C.c_void_p(ids.ctypes.data), C.c_void_p(out.ctypes.data)
    assert L.vcbct_organs_to_elements(ip, 0, 1, C.byref(t), op, 0, None) == ARG
    assert L.vcbct_organs_to_elements(ip, 4, 70000, C.byref(t), op, 0, None) == LIMIT


def test_file_readers_report_missing_files(L, tmp_path):
    d = N.ProjDeckC()
    assert L.vcbct_proj_deck_read(str(tmp_path / "none.txt").encode(), C.byref(d)) == IO
    assert "not found" in _msg(L)
    fd = N.FdkDeckC()
    assert L.vcbct_fdk_deck_read(str(tmp_path / "none.txt").encode(), C.byref(fd)) == IO
    n = C.c_int()
    assert L.vcbct_flexmap_read(str(tmp_path / "none.flexmap").encode(), 0, None, None, None, C.byref(n)) == IO
    t = N.PhantomTablesC()
    assert L.vcbct_phantom_tables_read(str(tmp_path / "m.csv").encode(), str(tmp_path / "o.csv").encode(), 1,
                                       C.byref(t)) == IO
    (tmp_path / "m.csv").write_text("1,2,3\n")                 # a row with too few columns
    (tmp_path / "o.csv").write_text("1,1,1.0\n")
    assert L.vcbct_phantom_tables_read(str(tmp_path / "m.csv").encode(), str(tmp_path / "o.csv").encode(), 1,
                                       C.byref(t)) == IO
    assert "malformed" in _msg(L)
