"""Geometry records and host-side table preparation.

Mirrors the reference's compile-time geometry (``physParams.h`` of both
programs) as runtime records, and its per-view table builder
``prepareTrigonometricTable`` (Release_CBCT_Projection_CM/misc.cpp:10-37),
which runs in the C library.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, fields, replace

import numpy as np

from . import _native as N

# Release_CBCT_Projection_CM/physParams.h:47-51 ("400 400 CBCT geometry CM")
DETECTOR_PITCH_CM_kV = 0.05
DETECTOR_PITCH_CM_AT_ISO_CENT_kV = 0.032509752
DIST_BTWN_SRC_AND_ISOCENT_CM_kV = 100.0
DETECTOR_PIXEL_NUM_kV = 800.0
DIST_BTWN_DETECTOR_AND_ISOCENT_CM_kV = 53.8


@dataclass(frozen=True)
class ProjGeometry:
    """Arguments of ``initializeGPU`` (reprojectionOnGPU.h:2-8)."""
    N: int                      # reconSize
    Z: int                      # reconSlices (usedZNumber)
    s: float                    # reconScale [cm]
    step: float                 # reconStep [cm]
    W: int                      # projImgWidth
    H: int                      # projImgHeight
    V: int                      # number of views
    pdet: float = DETECTOR_PITCH_CM_kV
    piso: float = DETECTOR_PITCH_CM_AT_ISO_CENT_kV
    sad: float = DIST_BTWN_SRC_AND_ISOCENT_CM_kV
    dpn: float = DETECTOR_PIXEL_NUM_kV
    x_reg: float = 0.0
    y_reg: float = 0.0
    z_reg: float = 0.0
    nmat: int = 6

    def to_c(self) -> N.ProjGeometryC:
        return N.ProjGeometryC(self.N, self.Z, self.s, self.step, self.W, self.H, self.V,
                               self.pdet, self.piso, self.sad, self.dpn, self.x_reg,
                               self.y_reg, self.z_reg, self.nmat)

    def with_(self, **kw) -> "ProjGeometry":
        return replace(self, **kw)


@dataclass(frozen=True)
class FdkGeometry:
    """Geometry of filterSinogram/reconstructImage; the reference's compile-time
    constants (R/physParams.h:22-41) are fields with the reference's values."""
    W: int = 400
    H: int = 400
    V: int = 36
    N: int = 270
    Z: int = 50
    zstart: int = -5
    step: float = 0.2
    scale: float = 0.1
    xfactor: int = 1000
    piso: float = 0.032509752
    pdet: float = 0.05
    mpn: float = 800.0
    sad: float = 100.0
    cutoff: float = 1.60
    gamma: float = 1.00
    alpha: float = 0.50
    redundancy: int = 0

    def to_c(self) -> N.FdkGeometryC:
        return N.FdkGeometryC(self.W, self.H, self.V, self.N, self.Z, self.zstart, self.step,
                              self.scale, self.xfactor, self.piso, self.pdet, self.mpn, self.sad,
                              self.cutoff, self.gamma, self.alpha, self.redundancy)

    def with_(self, **kw) -> "FdkGeometry":
        return replace(self, **kw)


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def trig_tables(W: int, H: int, angles_rad, xshift, yshift, pdet=DETECTOR_PITCH_CM_kV,
                dpn=DETECTOR_PIXEL_NUM_kV):
    """prepareTrigonometricTable (misc.cpp:10-37): (cos, sin, Xc, Yc) per view."""
    a = np.ascontiguousarray(angles_rad, np.float64)
    xs = np.ascontiguousarray(xshift, np.float64)
    ys = np.ascontiguousarray(yshift, np.float64)
    V = a.shape[0]
    out = [np.zeros(V, np.float64) for _ in range(4)]
    N.check(N.lib().vcbct_proj_trig_tables(W, H, V, _dptr(a), _dptr(xs), _dptr(ys), pdet, dpn,
                                           *[_dptr(o) for o in out]))
    return tuple(out)


def attenuation_table(spectrum_csv: str, xraydb_dir: str, nmat: int = 6, nthin: int = 1):
    """attenuation_coefficient (prior_weight_production.cpp:200-523):
    returns (mu float32 [nmat][NE] in cm^2/g, pdf float32 [NE])."""
    mu = np.zeros(nmat * N.MAX_BINS, np.float32)
    pdf = np.zeros(N.MAX_BINS, np.float32)
    ne = C.c_int(0)
    N.check(N.lib().vcbct_attenuation_table(spectrum_csv.encode(), xraydb_dir.encode(), nmat,
                                            nthin, mu.ctypes.data_as(C.POINTER(C.c_float)),
                                            pdf.ctypes.data_as(C.POINTER(C.c_float)),
                                            C.byref(ne)))
    n = ne.value
    return mu[: nmat * n].reshape(nmat, n).copy(), pdf[:n].copy()


__all__ = ["ProjGeometry", "FdkGeometry", "trig_tables", "attenuation_table", "fields"]
