"""ctypes binding of libvcbct.so (the C ABI declared in include/vcbct.h).

The library is built in-tree by ``virtualcbct_b200/csrc/Makefile`` (see
``__graft_entry__.build``).  There is no fallback: if the library is missing,
``lib()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvcbct.so")

VCBCT_OK = 0
ERRORS = {1: "invalid argument", 2: "CUDA error", 3: "limit exceeded", 4: "bad state",
          5: "I/O error", 6: "device fault flag"}

MAX_MATERIALS = 8
MAX_BINS = 1024

FILTER_DIRECT_F32 = 0
FILTER_BF16X3 = 1


class VcbctError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"vcbct error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class ProjGeometryC(C.Structure):
    _fields_ = [("recon_size", C.c_int), ("recon_slices", C.c_int),
                ("recon_scale", C.c_double), ("recon_step", C.c_double),
                ("proj_width", C.c_int), ("proj_height", C.c_int), ("n_views", C.c_int),
                ("det_pitch_cm", C.c_double), ("det_pitch_iso_cm", C.c_double),
                ("sad_cm", C.c_double), ("det_pixel_num", C.c_double),
                ("x_reg", C.c_double), ("y_reg", C.c_double), ("z_reg", C.c_double),
                ("num_material", C.c_int)]


class FdkGeometryC(C.Structure):
    _fields_ = [("proj_width", C.c_int), ("proj_height", C.c_int), ("n_views", C.c_int),
                ("recon_size", C.c_int), ("recon_slices", C.c_int), ("zstart", C.c_int),
                ("recon_step", C.c_double), ("recon_scale", C.c_double), ("xfactor", C.c_int),
                ("det_pitch_iso_cm", C.c_double), ("det_pitch_cm", C.c_double),
                ("max_pic_num", C.c_double), ("sad_cm", C.c_double), ("cutoff", C.c_double),
                ("gamma", C.c_double), ("alpha", C.c_double), ("redundancy", C.c_int)]


FDK_MAX_VIEWS = 1080


class ProjDeckC(C.Structure):
    """vcbct_proj_deck (the projector's info file)."""
    _fields_ = [("spectrum", C.c_char * 256), ("total_proj", C.c_int), ("proj_width", C.c_int),
                ("proj_height", C.c_int), ("angle_file", C.c_char * 256), ("mat_prefix", C.c_char * 256),
                ("z_ic", C.c_int), ("output_name", C.c_char * 256), ("x_scale", C.c_double),
                ("y_scale", C.c_double), ("z_scale", C.c_double), ("recon_size", C.c_int),
                ("recon_slices", C.c_int), ("mat_num", C.c_int), ("mat_type", C.c_char * 16),
                ("xfactor", C.c_double), ("x_reg", C.c_double), ("y_reg", C.c_double),
                ("z_reg_file", C.c_double), ("det_pitch_cm", C.c_double), ("det_pitch_iso_cm", C.c_double),
                ("sad_cm", C.c_double), ("det_pixel_num", C.c_double), ("det_iso_cm", C.c_double),
                ("slice_first", C.c_int), ("used_slices", C.c_int), ("z_ic_local", C.c_int),
                ("z_reg", C.c_double)]


class FdkDeckC(C.Structure):
    """vcbct_fdk_deck (the FDK info file and its flexmap)."""
    _fields_ = [("energy_class", C.c_char * 16), ("total_proj", C.c_int), ("proj_width", C.c_int),
                ("proj_height", C.c_int), ("proj_header_bytes", C.c_int), ("proj_prefix", C.c_char * 256),
                ("proj_num_digits", C.c_int), ("proj_first_number", C.c_int), ("proj_ext", C.c_char * 8),
                ("angle_file", C.c_char * 256), ("recon_size", C.c_int), ("target_class", C.c_char * 16),
                ("recon_offset", C.c_int), ("recon_step", C.c_double), ("recon_slices", C.c_int),
                ("recon_scale", C.c_double), ("xfactor", C.c_int), ("recon_file", C.c_char * 256),
                ("det_pitch_iso_cm", C.c_double), ("n_lines", C.c_int), ("n_target", C.c_int),
                ("reversed", C.c_int), ("panel_class", C.c_char * 8),
                ("angles_rad", C.c_double * FDK_MAX_VIEWS), ("xshift", C.c_double * FDK_MAX_VIEWS),
                ("yshift", C.c_double * FDK_MAX_VIEWS)]


class PhantomTablesC(C.Structure):
    """vcbct_phantom_tables."""
    _fields_ = [("n_media", C.c_int), ("n_organs", C.c_int), ("media_id", C.c_int * 100),
                ("media", (C.c_float * 6) * 100), ("organ", C.c_int * 150), ("organ_medium", C.c_int * 150),
                ("organ_density", C.c_float * 150), ("table", (C.c_uint16 * 6) * 256)]


_vp = C.c_void_p
_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)

# Every extern "C" symbol of include/vcbct.h with its ctypes signature.
SIGNATURES = {
    "vcbct_last_error": (C.c_char_p, []),
    "vcbct_version": (C.c_char_p, []),
    "vcbct_projector_create": (C.c_int, [C.POINTER(ProjGeometryC), _dp, _dp, _dp, _dp, C.POINTER(_vp)]),
    "vcbct_projector_destroy": (C.c_int, [_vp]),
    "vcbct_projector_set_spectrum": (C.c_int, [_vp, _fp, _fp, C.c_int, C.c_double]),
    "vcbct_projector_load_volume": (C.c_int, [_vp, _vp, C.c_int, _vp]),
    "vcbct_projector_load_volume_f32": (C.c_int, [_vp, _vp, C.c_int, _vp]),
    "vcbct_projector_forward": (C.c_int, [_vp, _vp, C.c_int, _vp]),
    "vcbct_projector_project": (C.c_int, [_vp, _vp, _vp, _vp]),
    "vcbct_projector_path_integrals": (C.c_int, [_vp, _vp, _vp]),
    "vcbct_projector_count_segments": (C.c_int, [_vp, C.POINTER(C.c_ulonglong), _vp]),
    "vcbct_projector_adjoint": (C.c_int, [_vp, _vp, _vp, _vp]),
    "vcbct_projector_forward_state": (C.c_int, [_vp, _vp, _vp, _vp]),
    "vcbct_projector_adjoint_state": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "vcbct_batch_create": (C.c_int, [C.POINTER(_vp)]),
    "vcbct_batch_add": (C.c_int, [_vp, _vp, _vp]),
    "vcbct_batch_forward": (C.c_int, [_vp, C.c_int, _vp]),
    "vcbct_batch_destroy": (C.c_int, [_vp]),
    "vcbct_batch_configure": (C.c_int, [_vp, C.c_int, C.c_int]),
    "vcbct_projector_autotune": (C.c_int, [_vp, _vp, _vp, _ip]),
    "vcbct_batch_autotune": (C.c_int, [_vp, _vp, _ip]),
    "vcbct_mbfpa_forward_noalloc": (C.c_int, [C.POINTER(ProjGeometryC), _dp, _dp, _dp, _dp, _vp, _fp,
                                              _fp, C.c_int, C.c_double, _vp, _vp]),
    "vcbct_projector_set_noise": (C.c_int, [_vp, C.c_int, C.c_double, C.c_double, C.c_ulonglong]),
    "vcbct_gaussian_noise": (C.c_int, [_vp, C.c_size_t, C.c_double, C.c_ulonglong, C.c_int, _vp]),
    "vcbct_philox4x32_10": (None, [_vp, _vp, _vp]),
    "vcbct_projector_lengthproj": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp]),
    "vcbct_ir_update": (C.c_int, [C.c_int, C.c_int, C.c_double, _vp, _vp, _vp, _vp, C.c_double, C.c_double,
                                  C.c_double, C.c_int, _vp]),
    "vcbct_lengthproj": (None, [C.c_int, C.c_int, C.c_int, _vp, _vp, _fp, _vp, C.c_double, C.c_double, C.c_int,
                          C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_double, _dp, C.c_double,
                          C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double]),
    "vcbct_IR_ImageCBCT": (None, [C.c_int, C.c_int, C.c_int, C.c_double, _vp, _fp, _fp, _fp, C.c_double, C.c_double,
                            C.c_double, C.c_int]),
    "vcbct_proj_trig_tables": (C.c_int, [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, C.c_double,
                                         C.c_double, _dp, _dp, _dp, _dp]),
    "vcbct_attenuation_table": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_int, _fp, _fp, _ip]),
    "vcbct_proj_deck_read": (C.c_int, [C.c_char_p, C.POINTER(ProjDeckC)]),
    "vcbct_proj_deck_load_volume": (C.c_int, [C.POINTER(ProjDeckC), _vp, _ip]),
    "vcbct_projector_load_deck": (C.c_int, [_vp, C.POINTER(ProjDeckC), _ip, _vp]),
    "vcbct_flexmap_read": (C.c_int, [C.c_char_p, C.c_int, _dp, _dp, _dp, _ip]),
    "vcbct_fdk_deck_read": (C.c_int, [C.c_char_p, C.POINTER(FdkDeckC)]),
    "vcbct_phantom_tables_read": (C.c_int, [C.c_char_p, C.c_char_p, C.c_uint, C.POINTER(PhantomTablesC)]),
    "vcbct_organs_to_elements": (C.c_int, [_vp, C.c_longlong, C.c_int, C.POINTER(PhantomTablesC), _vp, C.c_int,
                                           _vp]),
    "vcbct_fdk_default_geometry": (None, [C.POINTER(FdkGeometryC)]),
    "vcbct_fdk_create": (C.c_int, [C.POINTER(FdkGeometryC), _dp, _dp, _dp, C.POINTER(_vp)]),
    "vcbct_fdk_destroy": (C.c_int, [_vp]),
    "vcbct_fdk_redundancy_weights": (C.c_int, [C.POINTER(FdkGeometryC), _dp, _fp]),
    "vcbct_fdk_set_kernel": (C.c_int, [_vp, _dp]),
    "vcbct_fdk_filter": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_int, _vp]),
    "vcbct_fdk_backproject": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, _vp]),
    # C-linkage twins of the reference-named entry points
    "vcbct_initializeGPU": (None, [C.c_int, C.c_double, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int,
                             _dp, _dp, _dp, _dp, C.c_double, C.c_double, C.c_double, C.c_double,
                             C.c_double, C.c_double, C.c_double, C.c_int]),
    "vcbct_terminateGPU": (None, []),
    "vcbct_reprojectionOnGPU": (None, [C.c_int, C.c_int, C.c_int, _vp, _fp, _fp, _fp, C.c_double,
                                 C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp,
                                 _dp, _dp, C.c_double, _dp, C.c_double, C.c_double, C.c_double,
                                 C.c_double, C.c_double, C.c_double, C.c_double, _fp, _fp,
                                 C.c_int, C.c_int, C.c_char_p]),
    "vcbct_prepareConstMap": (C.POINTER(_dp), [C.c_int, C.c_double]),
    "vcbct_free_const_map": (None, [C.POINTER(_dp), C.c_int]),
    "vcbct_filterSinogram": (None, [C.c_int, C.c_int, C.c_int, _vp, _vp, C.POINTER(_dp), _dp, _dp,
                              C.c_double]),
    "vcbct_reconstructImage": (None, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _vp, _vp,
                                C.c_int, C.c_int, C.c_int, _vp, C.c_int, _dp, _dp, _dp, _dp,
                                C.c_double]),
}

_lock = threading.Lock()
_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    """Load libvcbct.so (once).  Raises if it has not been built."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `make -C virtualcbct_b200/csrc` "
                "(or __graft_entry__.build()); there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
        return L


def check(rc: int) -> None:
    if rc != VCBCT_OK:
        msg = lib().vcbct_last_error()
        raise VcbctError(rc, msg.decode() if msg else "")
