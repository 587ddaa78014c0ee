"""TEST INFRASTRUCTURE ONLY: ctypes bindings of the CPU oracle.

See ``oracle/__init__.py``.  Each wrapper names the reference function it
stands for; the C side (``vcbct_oracle.c`` / ``ref_driver.cpp``) cites the
reference file and line of every step.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LOCK = threading.Lock()
_LIBS: dict[str, C.CDLL] = {}

TIES_GPU = 0
TIES_CPU = 1

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_i64p = C.POINTER(C.c_int64)
_u16p = C.POINTER(C.c_uint16)


class OrcProjGeom(C.Structure):
    _fields_ = [("N", C.c_int), ("Z", C.c_int), ("s", C.c_double), ("step", C.c_double),
                ("W", C.c_int), ("H", C.c_int), ("V", C.c_int),
                ("pdet", C.c_double), ("piso", C.c_double), ("sad", C.c_double),
                ("dpn", C.c_double), ("x_reg", C.c_double), ("y_reg", C.c_double),
                ("z_reg", C.c_double), ("nmat", C.c_int)]


class OrcFdkConsts(C.Structure):
    _fields_ = [("mpn", C.c_double), ("pdet", C.c_double), ("sad", C.c_double),
                ("piso", C.c_double), ("cutoff", C.c_double), ("gamma_", C.c_double),
                ("alpha", C.c_double)]


def _ptr(a, t):
    if a is None:
        return None
    return a.ctypes.data_as(t)


def _load(name: str) -> C.CDLL:
    with _LOCK:
        if name in _LIBS:
            return _LIBS[name]
        path = os.path.join(HERE, name)
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", HERE], check=False)
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library {path} is not built")
        lib = C.CDLL(path, mode=C.RTLD_LOCAL)
        _LIBS[name] = lib
        return lib


@contextlib.contextmanager
def quiet_stdout():
    """Send the process's C-level stdout (fd 1) to /dev/null for the
    duration: the reference's CPU code prints progress lines there, which
    must not mix with a caller's own output (bench.py prints one JSON line)."""
    libc = C.CDLL(None)
    libc.fflush(None)
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    try:
        os.dup2(devnull, 1)
        yield
    finally:
        libc.fflush(None)
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)


def have_reference() -> bool:
    """True when the reference's own CPU code (oracle/_ref) is built."""
    return all(os.path.exists(os.path.join(HERE, "_ref", n))
               for n in ("libref_proj.so", "libref_fdk.so"))


def lib():
    return _load("liboracle.so")


# ----------------------------------------------------------------- geometry --

def proj_geom(g) -> OrcProjGeom:
    """Build the C struct from any object with the projector geometry fields."""
    return OrcProjGeom(g.N, g.Z, g.s, g.step, g.W, g.H, g.V, g.pdet, g.piso, g.sad,
                       g.dpn, g.x_reg, g.y_reg, g.z_reg, g.nmat)


def trig_tables(W, H, angles_rad, xshift, yshift, pdet, dpn):
    """P/misc.cpp:10-37 prepareTrigonometricTable (restated)."""
    V = len(angles_rad)
    a = np.ascontiguousarray(angles_rad, np.float64)
    xs = np.ascontiguousarray(xshift, np.float64)
    ys = np.ascontiguousarray(yshift, np.float64)
    out = [np.zeros(V, np.float64) for _ in range(4)]
    L = lib()
    L.orc_trig_tables.restype = None
    L.orc_trig_tables(C.c_int(W), C.c_int(H), C.c_int(V), _ptr(a, _dp), _ptr(xs, _dp),
                      _ptr(ys, _dp), C.c_double(pdet), C.c_double(dpn),
                      *[_ptr(o, _dp) for o in out])
    return tuple(out)


# -------------------------------------------------------------------- MBFPA --

def mbfpa_forward(g, tables, vol, mu, pdf, xfactor, views=None, rows=None, cols=None,
                  ties=TIES_GPU, with_leng=True, flip=True, exact=True, volf=None,
                  want=("f",)):
    """Restated reprojectionKernel + host energy loop (P/reprojectionOnGPU.cu:56-1056).

    vol: uint16 [Z][nmat][N][N]; volf (float32, same layout) replaces it.
    mu: float32 [nmat][NE]; pdf: float32 [NE].
    want: any of "f" (float-summed reference output), "d" (FP64), "L" (per
    element path integrals), "nb"/"nm" (segment counts).  Returns a dict.
    """
    gc = proj_geom(g)
    V, H, W = g.V, g.H, g.W
    cosT, sinT, Xc, Yc = [np.ascontiguousarray(t, np.float64) for t in tables]
    views = np.arange(V, dtype=np.int32) if views is None else np.ascontiguousarray(views, np.int32)
    j0, j1 = (0, H) if rows is None else rows
    c0, c1 = (0, W) if cols is None else cols
    mu = np.ascontiguousarray(mu, np.float32)
    pdf = np.ascontiguousarray(pdf, np.float32)
    NE = int(pdf.shape[0])
    res = {}
    if "f" in want:
        res["f"] = np.zeros((V, H, W), np.float32)
    if "d" in want:
        res["d"] = np.zeros((V, H, W), np.float64)
    if "L" in want:
        res["L"] = np.zeros((V, H, W, g.nmat), np.float64)
    if "nb" in want:
        res["nb"] = np.zeros((V, H, W), np.int64)
    if "nm" in want:
        res["nm"] = np.zeros((V, H, W), np.int64)
    vol_p = None if vol is None else _ptr(np.ascontiguousarray(vol, np.uint16), _u16p)
    volf_c = None if volf is None else np.ascontiguousarray(volf, np.float32)
    L = lib()
    L.orc_mbfpa_forward.restype = C.c_int
    rc = L.orc_mbfpa_forward(
        C.byref(gc), _ptr(cosT, _dp), _ptr(sinT, _dp), _ptr(Xc, _dp), _ptr(Yc, _dp),
        vol_p, _ptr(volf_c, _fp), _ptr(mu, _fp), _ptr(pdf, _fp), C.c_int(NE),
        C.c_double(xfactor), _ptr(views, _ip), C.c_int(len(views)),
        C.c_int(j0), C.c_int(j1), C.c_int(c0), C.c_int(c1), C.c_int(ties),
        C.c_int(int(with_leng)), C.c_int(int(flip)), C.c_int(int(exact)),
        _ptr(res.get("f"), _fp), _ptr(res.get("d"), _dp), _ptr(res.get("L"), _dp),
        _ptr(res.get("nb"), _i64p), _ptr(res.get("nm"), _i64p))
    if rc != 0:
        raise ValueError(f"orc_mbfpa_forward failed ({rc})")
    return res


def mbfpa_adjoint(g, tables, volf, mu, pdf, xfactor, resid):
    """FP64 gradient of sum(resid * I) w.r.t. float element volumes."""
    gc = proj_geom(g)
    cosT, sinT, Xc, Yc = [np.ascontiguousarray(t, np.float64) for t in tables]
    volf = np.ascontiguousarray(volf, np.float32)
    grad = np.zeros(volf.shape, np.float64)
    resid = np.ascontiguousarray(resid, np.float64)
    mu = np.ascontiguousarray(mu, np.float32)
    pdf = np.ascontiguousarray(pdf, np.float32)
    L = lib()
    L.orc_mbfpa_adjoint.restype = C.c_int
    rc = L.orc_mbfpa_adjoint(C.byref(gc), _ptr(cosT, _dp), _ptr(sinT, _dp), _ptr(Xc, _dp),
                             _ptr(Yc, _dp), _ptr(volf, _fp), _ptr(mu, _fp), _ptr(pdf, _fp),
                             C.c_int(int(pdf.shape[0])), C.c_double(xfactor),
                             _ptr(resid, _dp), _ptr(grad, _dp))
    if rc != 0:
        raise ValueError("orc_mbfpa_adjoint failed")
    return grad


# ---------------------------------------------------------------------- FDK --

def fdk_consts(piso, mpn=800.0, pdet=0.05, sad=100.0, cutoff=1.6, gamma_=1.0, alpha=0.5):
    return OrcFdkConsts(mpn, pdet, sad, piso, cutoff, gamma_, alpha)


def const_map(W, consts):
    """R/filterSinogram.cpp:10-65 prepareConstMap (restated)."""
    h = np.zeros((W, W), np.float64)
    L = lib()
    L.orc_const_map.restype = None
    L.orc_const_map(C.c_int(W), C.byref(consts), _ptr(h, _dp))
    return h


def filter_coeff(W, consts):
    L = lib()
    L.orc_filter_coeff.restype = C.c_double
    return L.orc_filter_coeff(C.c_int(W), C.byref(consts))


def filter_sinogram(proj, xshift, yshift, consts, mode=0, h=None):
    """R/filterSinogram.cpp:67-131 (restated).  mode 0: float accumulation
    (reference), mode 1: FP64 accumulation (returns float64)."""
    proj = np.ascontiguousarray(proj, np.float32)
    V, H, W = proj.shape
    if h is None:
        h = const_map(W, consts)
    xs = np.ascontiguousarray(xshift, np.float64)
    ys = np.ascontiguousarray(yshift, np.float64)
    out_f = np.zeros(proj.shape, np.float32) if mode == 0 else None
    out_d = np.zeros(proj.shape, np.float64) if mode == 1 else None
    L = lib()
    L.orc_filter.restype = None
    L.orc_filter(C.c_int(V), C.c_int(H), C.c_int(W), _ptr(proj, _fp),
                 _ptr(np.ascontiguousarray(h, np.float64), _dp), _ptr(xs, _dp), _ptr(ys, _dp),
                 C.byref(consts), C.c_int(mode), _ptr(out_f, _fp), _ptr(out_d, _dp))
    return out_f if mode == 0 else out_d


def mask(N):
    m = np.zeros((N, N), np.int8)
    L = lib()
    L.orc_mask.restype = None
    L.orc_mask(C.c_int(N), m.ctypes.data_as(C.c_char_p))
    return m


def backproject(N, Z, zstart, step, scale, filt, xfactor, angles, xshift, consts,
                vol=None):
    """R/reconstructImage.cpp:10-184 (restated); returns the double volume."""
    filt_f = filt_d = None
    if filt.dtype == np.float64:
        filt_d = np.ascontiguousarray(filt)
    else:
        filt_f = np.ascontiguousarray(filt, np.float32)
    V, H, W = filt.shape
    angles = np.ascontiguousarray(angles, np.float64)
    cosT = np.cos(angles)
    sinT = np.sin(angles)
    xs = np.ascontiguousarray(xshift, np.float64)
    m = mask(N)
    out = np.zeros((Z, N, N), np.float64) if vol is None else np.ascontiguousarray(vol, np.float64)
    L = lib()
    L.orc_backproject.restype = None
    L.orc_backproject(C.c_int(N), C.c_int(Z), C.c_int(zstart), C.c_double(step),
                      C.c_double(scale), _ptr(out, _dp), m.ctypes.data_as(C.c_char_p),
                      C.c_int(H), C.c_int(W), C.c_int(V), _ptr(filt_f, _fp), _ptr(filt_d, _dp),
                      C.c_int(int(xfactor)), _ptr(angles, _dp), _ptr(cosT, _dp), _ptr(sinT, _dp),
                      _ptr(xs, _dp), C.byref(consts))
    return out


# -------------------------------------------------- the reference's own code --

def ref_proj():
    return _load(os.path.join("_ref", "libref_proj.so"))


def ref_fdk():
    return _load(os.path.join("_ref", "libref_fdk.so"))


def ref_mbfpa_views(g, tables, vol, mu, pdf, xfactor, views, bins, nthreads=0):
    """Reference CPU twin reprojection() (P/reprojection.cpp:10) driven per
    (view, bin); returns (float [V][H][W] un-flipped, no cos^3, seconds)."""
    L = ref_proj()
    L.ref_mbfpa_views.restype = C.c_double
    cosT, sinT, Xc, Yc = [np.ascontiguousarray(t, np.float64) for t in tables]
    vol = np.ascontiguousarray(vol, np.uint16)
    mu = np.ascontiguousarray(mu, np.float32)
    pdf = np.ascontiguousarray(pdf, np.float32)
    views = np.ascontiguousarray(views, np.int32)
    bins = np.ascontiguousarray(bins, np.int32)
    out = np.zeros((g.V, g.H, g.W), np.float32)
    secs = L.ref_mbfpa_views(
        C.c_int(g.N), C.c_int(g.Z), _ptr(vol, _u16p), C.c_double(g.s), C.c_double(g.step),
        C.c_int(g.W), C.c_int(g.H), _ptr(cosT, _dp), _ptr(sinT, _dp), _ptr(Xc, _dp),
        _ptr(Yc, _dp), C.c_double(xfactor), C.c_double(g.pdet), C.c_double(g.piso),
        C.c_double(g.sad), C.c_double(g.dpn), C.c_double(g.x_reg), C.c_double(g.y_reg),
        C.c_double(g.z_reg), _ptr(mu, _fp), _ptr(pdf, _fp), C.c_int(g.nmat),
        C.c_int(int(pdf.shape[0])), _ptr(views, _ip), C.c_int(len(views)), _ptr(bins, _ip),
        C.c_int(len(bins)), C.c_int(nthreads), _ptr(out, _fp))
    return out, secs


def ref_trig_tables(W, H, angles_rad, xshift, yshift, pdet, dpn):
    """The reference's own prepareTrigonometricTable (P/misc.cpp:10-37)."""
    L = ref_proj()
    L.ref_proj_trig.restype = C.c_int
    a = np.ascontiguousarray(angles_rad, np.float64)
    xs = np.ascontiguousarray(xshift, np.float64)
    ys = np.ascontiguousarray(yshift, np.float64)
    V = a.shape[0]
    out = [np.zeros(V, np.float64) for _ in range(4)]
    L.ref_proj_trig(C.c_int(W), C.c_int(H), C.c_int(V), _ptr(a, _dp), _ptr(xs, _dp), _ptr(ys, _dp),
                    C.c_double(pdet), C.c_double(dpn), *[_ptr(o, _dp) for o in out])
    return tuple(out)


def mbfpa_sampled(g, tables, vol, mu, pdf, xfactor, views, cols, want=("d",), **kw):
    """mbfpa_forward on a sample of rays: the given views and detector
    columns, every row (or the detector rows `rows=(j0, j1)`).  Returns each
    output of `want` as [len(views)][H][len(cols)] (rows in the output
    layout: flipped unless flip=False; rows outside a given range are 0)."""
    views = np.ascontiguousarray(views, np.int32)
    cols = np.asarray(cols, np.int32)
    res = {k: np.zeros((len(views), g.H, len(cols)), np.float64 if k != "f" else np.float32) for k in want}
    pos = {int(c): i for i, c in enumerate(cols)}
    start = 0
    while start < len(cols):
        end = start
        while end + 1 < len(cols) and cols[end + 1] == cols[end] + 1:
            end += 1
        c0, c1 = int(cols[start]), int(cols[end]) + 1
        r = mbfpa_forward(g, tables, vol, mu, pdf, xfactor, views=views, cols=(c0, c1), want=want, **kw)
        for k in want:
            res[k][:, :, pos[c0]:pos[c0] + (c1 - c0)] = r[k][views][:, :, c0:c1]
        start = end + 1
    return res


def ref_attenuation(workdir, spectrum, nmat, mat_type="human"):
    """Reference attenuation_coefficient (P/prior_weight_production.cpp:200)."""
    L = ref_proj()
    L.ref_attenuation.restype = C.c_int
    mu = np.zeros(1024 * nmat, np.float32)
    pdf = np.zeros(1024, np.float32)
    with quiet_stdout():
        NE = L.ref_attenuation(workdir.encode(), spectrum.encode(), C.c_int(nmat),
                               mat_type.encode(), _ptr(mu, _fp), _ptr(pdf, _fp))
    if NE <= 0:
        raise RuntimeError("reference attenuation_coefficient failed")
    return mu[: nmat * NE].reshape(nmat, NE).copy(), pdf[:NE].copy()


def ref_filter(proj, xshift, yshift, piso, nthreads=0):
    """Reference filterSinogram (R/filterSinogram.cpp:67); (out, seconds)."""
    L = ref_fdk()
    L.ref_filter.restype = C.c_double
    proj = np.ascontiguousarray(proj, np.float32)
    V, H, W = proj.shape
    out = np.zeros_like(proj)
    secs = L.ref_filter(C.c_int(V), C.c_int(H), C.c_int(W), _ptr(proj, _fp), _ptr(out, _fp),
                        _ptr(np.ascontiguousarray(xshift, np.float64), _dp),
                        _ptr(np.ascontiguousarray(yshift, np.float64), _dp),
                        C.c_double(piso), C.c_int(nthreads))
    return out, secs


def ref_backproject(N, Z, zstart, step, scale, filt, xfactor, angles, xshift, piso,
                    nthreads=0):
    """Reference reconstructImage (R/reconstructImage.cpp:10); (vol, seconds)."""
    L = ref_fdk()
    L.ref_backproject.restype = C.c_double
    filt = np.ascontiguousarray(filt, np.float32)
    V, H, W = filt.shape
    vol = np.zeros((Z, N, N), np.float64)
    secs = L.ref_backproject(C.c_int(N), C.c_int(Z), C.c_int(zstart), C.c_double(step),
                             C.c_double(scale), _ptr(vol, _dp), C.c_int(H), C.c_int(W),
                             C.c_int(V), _ptr(filt, _fp), C.c_int(int(xfactor)),
                             _ptr(np.ascontiguousarray(angles, np.float64), _dp),
                             _ptr(np.ascontiguousarray(xshift, np.float64), _dp),
                             C.c_double(piso), C.c_int(nthreads))
    return vol, secs


def ref_const_map(W, piso):
    L = ref_fdk()
    L.ref_const_map.restype = None
    h = np.zeros((W, W), np.float64)
    L.ref_const_map(C.c_int(W), C.c_double(piso), _ptr(h, _dp))
    return h


def ref_mask(N):
    L = ref_fdk()
    L.ref_mask.restype = None
    m = np.zeros((N, N), np.int8)
    L.ref_mask(C.c_int(N), m.ctypes.data_as(C.c_char_p))
    return m


def ref_proj_load(txt):
    """Reference loadData + loadProjectionData of the projector
    (P/projectionData.cpp:63-237), run in the current directory; returns a
    dict of the fields, the flexmap arrays and the assembled volume."""
    L = ref_proj()
    L.ref_proj_load.restype = C.c_int
    L.ref_free.restype = None
    ints = np.zeros(8, np.int32)
    dbls = np.zeros(12, np.float64)
    spec, outn, mtype = (C.create_string_buffer(256), C.create_string_buffer(256),
                         C.create_string_buffer(16))
    vol, ang, xs, ys = C.POINTER(C.c_uint16)(), _dp(), _dp(), _dp()
    r = L.ref_proj_load(txt.encode(), _ptr(ints, _ip), _ptr(dbls, _dp), spec, outn, mtype,
                        C.byref(vol), C.byref(ang), C.byref(xs), C.byref(ys))
    if r == 0:
        raise RuntimeError("reference loadData failed")
    V, N, nmat, used = int(ints[0]), int(ints[4]), int(ints[6]), int(ints[7])
    out = dict(total_proj=V, proj_width=int(ints[1]), proj_height=int(ints[2]),
               z_ic_local=int(ints[3]), recon_size=N, recon_slices=int(ints[5]), mat_num=nmat,
               used_slices=used, x_scale=dbls[0], y_scale=dbls[1], z_scale=dbls[2],
               xfactor=dbls[3], x_reg=dbls[4], y_reg=dbls[5], z_reg_file=dbls[6],
               det_pitch_cm=dbls[7], det_pitch_iso_cm=dbls[8], sad_cm=dbls[9],
               det_pixel_num=dbls[10], det_iso_cm=dbls[11], spectrum=spec.value.decode(),
               output_name=outn.value.decode(), mat_type=mtype.value.decode())
    out["angles_rad"] = np.ctypeslib.as_array(ang, (V,)).copy()
    out["xshift"] = np.ctypeslib.as_array(xs, (V,)).copy()
    out["yshift"] = np.ctypeslib.as_array(ys, (V,)).copy()
    out["volume"] = np.ctypeslib.as_array(vol, (used * nmat * N * N,)).copy().reshape(used, nmat, N, N)
    for p in (vol, ang, xs, ys):
        L.ref_free(C.cast(p, C.c_void_p))
    return out


def ref_fdk_load(txt):
    """Reference loadData + loadProjectionData of the FDK program
    (R/projectionDataMVkV.cpp:51-321), run in the current directory."""
    L = ref_fdk()
    L.ref_fdk_load.restype = C.c_int
    ints = np.zeros(8, np.int32)
    dbls = np.zeros(3, np.float64)
    pdir, ext, outn, sml = (C.create_string_buffer(256), C.create_string_buffer(8),
                            C.create_string_buffer(256), C.create_string_buffer(8))
    ang, xs, ys = (np.zeros(1080), np.zeros(1080), np.zeros(1080))
    r = L.ref_fdk_load(txt.encode(), _ptr(ints, _ip), _ptr(dbls, _dp), pdir, ext, outn, sml,
                       _ptr(ang, _dp), _ptr(xs, _dp), _ptr(ys, _dp))
    used = int(ints[1])
    return dict(ret=int(r), n_target=int(ints[0]), total_proj=used, proj_width=int(ints[2]),
                proj_height=int(ints[3]), recon_size=int(ints[4]), recon_offset=int(ints[5]),
                recon_slices=int(ints[6]), xfactor=int(ints[7]), recon_step=dbls[0],
                recon_scale=dbls[1], det_pitch_iso_cm=dbls[2], proj_prefix=pdir.value.decode(),
                proj_ext=ext.value.decode(), recon_file=outn.value.decode(),
                panel_class=sml.value.decode(), angles_rad=ang[:used].copy(),
                xshift=xs[:used].copy(), yshift=ys[:used].copy())


# ------------------------------------------------------ iterative recon --

def lengthproj(g, tables, proj, ite=0, views=None):
    """P/lengthproj.cpp:10-131 restated; proj uint16 [V][H][W] -> float [Z][N][N]."""
    L = lib()
    L.orc_lengthproj.restype = None
    cosT, sinT, Xc, Yc = [np.ascontiguousarray(t, np.float64) for t in tables]
    v0, v1 = (0, g.V) if views is None else views
    proj = np.ascontiguousarray(proj, np.uint16)
    npf = np.zeros((g.Z, g.N, g.N), np.float32)
    L.orc_lengthproj(C.c_int(ite), C.c_int(g.N), C.c_int(g.Z), _ptr(proj, _u16p), _ptr(npf, _fp),
                     C.c_double(g.s), C.c_double(g.step), C.c_int(g.W), C.c_int(g.H), C.c_int(v0), C.c_int(v1),
                     _ptr(cosT, _dp), _ptr(sinT, _dp), _ptr(Xc, _dp), _ptr(Yc, _dp), C.c_double(g.pdet),
                     C.c_double(g.piso), C.c_double(g.sad), C.c_double(g.dpn), C.c_double(g.x_reg),
                     C.c_double(g.y_reg), C.c_double(g.z_reg))
    return npf


def ir_update(N, Z, scale, before, npf, npf_re, wbefore, wtv, wprior):
    """P/IR_ImageCBCT.cpp:10-93 restated."""
    L = lib()
    L.orc_ir_update.restype = None
    before = np.ascontiguousarray(before, np.int16)
    npf = np.ascontiguousarray(npf, np.float32)
    npf_re = np.ascontiguousarray(npf_re, np.float32)
    out = np.zeros((Z, N, N), np.float32)
    L.orc_ir_update(C.c_int(N), C.c_int(Z), C.c_double(scale), before.ctypes.data_as(C.POINTER(C.c_short)),
                    _ptr(out, _fp), _ptr(npf, _fp), _ptr(npf_re, _fp), C.c_double(wbefore), C.c_double(wtv),
                    C.c_double(wprior))
    return out


def ref_lengthproj(g, tables, proj, ite=0, views=None):
    """The reference's own lengthproj (compiled from P/lengthproj.cpp)."""
    L = ref_proj()
    L.ref_lengthproj.restype = None
    cosT, sinT, Xc, Yc = [np.ascontiguousarray(t, np.float64) for t in tables]
    v0, v1 = (0, g.V) if views is None else views
    proj = np.ascontiguousarray(proj, np.uint16)
    npf = np.zeros((g.Z, g.N, g.N), np.float32)
    L.ref_lengthproj(C.c_int(ite), C.c_int(g.N), C.c_int(g.Z), _ptr(proj, _u16p), _ptr(npf, _fp),
                     C.c_double(g.s), C.c_double(g.step), C.c_int(g.W), C.c_int(g.H), C.c_int(v0), C.c_int(v1),
                     _ptr(cosT, _dp), _ptr(sinT, _dp), _ptr(Xc, _dp), _ptr(Yc, _dp), C.c_double(g.pdet),
                     C.c_double(g.piso), C.c_double(g.sad), C.c_double(g.dpn), C.c_double(g.x_reg),
                     C.c_double(g.y_reg), C.c_double(g.z_reg))
    return npf


def ref_ir_update(N, Z, scale, before, npf, npf_re, wbefore, wtv, wprior):
    """The reference's own IR_ImageCBCT (compiled from P/IR_ImageCBCT.cpp)."""
    L = ref_proj()
    L.ref_ir_update.restype = None
    before = np.ascontiguousarray(before, np.int16).copy()
    npf = np.ascontiguousarray(npf, np.float32).copy()
    npf_re = np.ascontiguousarray(npf_re, np.float32).copy()
    out = np.zeros((Z, N, N), np.float32)
    L.ref_ir_update(C.c_int(N), C.c_int(Z), C.c_double(scale), before.ctypes.data_as(C.POINTER(C.c_short)),
                    _ptr(out, _fp), _ptr(npf, _fp), _ptr(npf_re, _fp), C.c_double(wbefore), C.c_double(wtv),
                    C.c_double(wprior))
    return out


def ref_gaussiannoise(proj, seed=1):
    """The reference's gaussiannoise (prior_weight_production.cpp:24-38)
    after srand(seed), on a copy of float proj (in its 65535-based units)."""
    L = ref_proj()
    L.ref_gaussiannoise.restype = None
    out = np.ascontiguousarray(proj, np.float32).copy()
    L.ref_gaussiannoise(_ptr(out, _fp), C.c_int(out.size), C.c_uint(seed))
    return out


def have_icrp_convert() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "icrp_convert"))


def ref_icrp_convert(workdir, organ_ids, media_csv, organs_csv):
    """Run the reference's converter (ICRPphantoms_2mmslice/
    To_material_distribution_for512_random.cpp, male branch) in `workdir` on
    an organ-number volume uint8 [100][271][543]; returns its element volume
    int16 [6][100][271][543] (the whole-volume test.raw it writes)."""
    import shutil
    organ_ids = np.ascontiguousarray(organ_ids, np.uint8)
    assert organ_ids.shape == (100, 271, 543)
    organ_ids.tofile(os.path.join(workdir, "AM_skin_543x271_700_800.raw"))
    shutil.copy(media_csv, os.path.join(workdir, "AM_media.csv"))
    shutil.copy(organs_csv, os.path.join(workdir, "AM_organs.csv"))
    os.makedirs(os.path.join(workdir, "AM_MD"), exist_ok=True)
    os.makedirs(os.path.join(workdir, "AM_ED"), exist_ok=True)
    subprocess.run([os.path.join(HERE, "_ref", "icrp_convert")], cwd=workdir, check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    return np.fromfile(os.path.join(workdir, "test.raw"), np.int16).reshape(6, 100, 271, 543)
