"""Host mirror of the FDK interface (filterSinogram + reconstructImage).

``Fdk`` owns a ``vcbct_fdk`` handle built from an ``FdkGeometry`` and the
per-view angle / shift lists in the order the projections are stored.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .geometry import FdkGeometry
from .projector import _is_torch_cuda, _stream_ptr


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def redundancy_weights(geom: FdkGeometry, xshift=None) -> np.ndarray:
    """The redundancy weights float [V][W] the filter applies to -log p when
    ``geom.redundancy`` is 1 (host computation, no device call)."""
    x = np.zeros(geom.V) if xshift is None else np.ascontiguousarray(xshift, np.float64)
    if x.shape[0] != geom.V:
        raise ValueError("xshift must have n_views entries")
    w = np.empty((geom.V, geom.W), np.float32)
    gc = geom.to_c()
    N.check(N.lib().vcbct_fdk_redundancy_weights(C.byref(gc), _dp(x),
                                                 w.ctypes.data_as(C.POINTER(C.c_float))))
    return w


class Fdk:
    def __init__(self, geom: FdkGeometry, angles_rad, xshift=None, yshift=None):
        self.geom = geom
        V = geom.V
        self._a = np.ascontiguousarray(angles_rad, np.float64)
        self._x = np.zeros(V) if xshift is None else np.ascontiguousarray(xshift, np.float64)
        self._y = np.zeros(V) if yshift is None else np.ascontiguousarray(yshift, np.float64)
        if self._a.shape[0] != V or self._x.shape[0] != V or self._y.shape[0] != V:
            raise ValueError("angle / shift lists must have n_views entries")
        h = C.c_void_p()
        gc = geom.to_c()
        N.check(N.lib().vcbct_fdk_create(C.byref(gc), _dp(self._a), _dp(self._x), _dp(self._y), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            N.lib().vcbct_fdk_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_kernel(self, h):
        h = np.ascontiguousarray(h, np.float64)
        if h.shape != (self.geom.W, self.geom.W):
            raise ValueError("ramp kernel must be [W][W]")
        N.check(N.lib().vcbct_fdk_set_kernel(self._h, _dp(h)))

    def filter(self, proj, out=None, method=N.FILTER_DIRECT_F32, stream=None):
        """filterSinogram: float [V][H][W] -> filtered float [V][H][W]."""
        g = self.geom
        L = N.lib()
        if _is_torch_cuda(proj):
            import torch
            p = proj.contiguous()
            if out is None:
                out = torch.empty_like(p)
            N.check(L.vcbct_fdk_filter(self._h, C.c_void_p(p.data_ptr()), C.c_void_p(out.data_ptr()), 1,
                                       int(method), _stream_ptr(stream)))
            return out
        p = np.ascontiguousarray(proj, np.float32)
        if p.shape != (g.V, g.H, g.W):
            raise ValueError("projections must be float32 [V][H][W]")
        out = np.empty_like(p) if out is None else out
        N.check(L.vcbct_fdk_filter(self._h, C.c_void_p(p.ctypes.data), C.c_void_p(out.ctypes.data), 0,
                                   int(method), None))
        return out

    def backproject(self, filtered, want_f32=True, want_i16=True, stream=None):
        """reconstructImage + the (short) cast: returns (vol_f32, vol_i16)."""
        g = self.geom
        L = N.lib()
        shape = (g.Z, g.N, g.N)
        if _is_torch_cuda(filtered):
            import torch
            f = filtered.contiguous()
            vf = torch.empty(shape, dtype=torch.float32, device=f.device) if want_f32 else None
            vi = torch.empty(shape, dtype=torch.int16, device=f.device) if want_i16 else None
            N.check(L.vcbct_fdk_backproject(self._h, C.c_void_p(f.data_ptr()),
                                            C.c_void_p(vf.data_ptr()) if vf is not None else None,
                                            C.c_void_p(vi.data_ptr()) if vi is not None else None,
                                            1, _stream_ptr(stream)))
            return vf, vi
        f = np.ascontiguousarray(filtered, np.float32)
        vf = np.empty(shape, np.float32) if want_f32 else None
        vi = np.empty(shape, np.int16) if want_i16 else None
        N.check(L.vcbct_fdk_backproject(self._h, C.c_void_p(f.ctypes.data),
                                        C.c_void_p(vf.ctypes.data) if vf is not None else None,
                                        C.c_void_p(vi.ctypes.data) if vi is not None else None, 0, None))
        return vf, vi

    def reconstruct(self, proj, method=N.FILTER_DIRECT_F32, stream=None):
        return self.backproject(self.filter(proj, method=method, stream=stream), stream=stream)
