"""Synthetic workloads of the benchmark configurations, shared by bench.py
and the parity tests so both run exactly the same inputs.

Self-contained (numpy only): the reference arm of bench.py builds its inputs
from here and from the reference's own code, without loading the product
library.  All inputs are deterministic, in the reference's formats: uint16
element volumes [Z][6][N][N] (density x mass fraction x 1000), spectra as
the reference's CSV, view angles as its flexmaps write them.
"""
from __future__ import annotations

import os
from dataclasses import asdict, dataclass

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
DATA = os.path.join(ROOT, "virtualcbct_b200", "data")
MINIDB = os.path.join(DATA, "xraydb_mini")
# the reference's projector directory as staged by oracle/Makefile (its
# attenuation_coefficient reads attenuation_xraydb/ relative to it)
REF_PROJ_DIR = os.path.join(ROOT, "oracle", "_ref", "data", "Release_CBCT_Projection_CM")

C2_NAME = ("25 cm water cylinder 512x512x200x6 u16 (0.5x0.5x2 mm), 360 views/1 deg, "
           "half-fan 160 px, 400x400 f32, 90-bin 100 kV; FDK 270x270x200")


@dataclass(frozen=True)
class Geometry:
    """The projector geometry (the arguments of initializeGPU,
    Release_CBCT_Projection_CM/reprojectionOnGPU.h:2-8), with the reference's
    compile-time detector constants (physParams.h:47-51) as defaults."""
    N: int
    Z: int
    s: float
    step: float
    W: int
    H: int
    V: int
    pdet: float = 0.05
    piso: float = 0.032509752
    sad: float = 100.0
    dpn: float = 800.0
    x_reg: float = 0.0
    y_reg: float = 0.0
    z_reg: float = 0.0
    nmat: int = 6

    def native(self):
        """The same geometry as the product's ProjGeometry."""
        from virtualcbct_b200 import ProjGeometry
        return ProjGeometry(**asdict(self))


@dataclass(frozen=True)
class FdkSetup:
    """The FDK geometry fields the workloads set (the rest keep the
    reference's R/physParams.h values)."""
    W: int
    H: int
    V: int
    N: int
    Z: int
    zstart: int
    step: float
    scale: float
    redundancy: int = 0

    def native(self, **kw):
        from virtualcbct_b200 import FdkGeometry
        return FdkGeometry(**{**asdict(self), **kw})


def view_angles(n_views: int, start_deg: float = -170.0001, span_deg: float = 360.0) -> np.ndarray:
    """Equally spaced view angles in degrees, the flexmap convention."""
    return start_deg + np.arange(n_views) * (span_deg / n_views)


def water_cylinder(N: int, Z: int, s: float, radius_cm: float) -> np.ndarray:
    """Uniform water cylinder along z, uint16 [Z][6][N][N]: H 111 and O 889
    (mass fractions 0.111 / 0.889 at 1 g/cm3, x1000) inside; outside, air as
    N = 1 (0.0012 g/cm3 x 1000, rounded, as the reference's phantom files)."""
    c = (np.arange(N) - (N - 1) / 2.0) * s
    inside = (c[None, :] ** 2 + c[:, None] ** 2) <= radius_cm ** 2
    vol = np.zeros((Z, 6, N, N), np.uint16)
    vol[:, 0] = np.where(inside, 111, 0)[None]
    vol[:, 2] = np.where(inside, 0, 1)[None]
    vol[:, 3] = np.where(inside, 889, 0)[None]
    return vol


def c2_workload(with_volume: bool = True) -> dict:
    """Plain MBFPA + FDK at scale: 25 cm water cylinder, 512x512x200 x 6
    elements (0.5 x 0.5 x 2 mm), 360 views at 1 deg with the half-fan offset
    (projector flexmap xshift 1.6 = 160 px; FDK flexmap 16), 400x400
    detector, 90-bin 100 kV filtered-Kramers spectrum; FDK to 270x270x200
    (1 mm) with the half-fan redundancy weights."""
    V, W, H = 360, 400, 400
    g = Geometry(N=512, Z=200, s=0.05, step=0.2, W=W, H=H, V=V)
    return dict(g=g, angles_deg=view_angles(V, -180.0001), xs_proj=np.full(V, 1.6), xs_fdk=np.full(V, 16.0),
                vol=water_cylinder(g.N, g.Z, g.s, 12.5) if with_volume else None,
                spectrum_csv=os.path.join(DATA, "spectrum_kramers100_90.csv"),
                fdk=FdkSetup(W=W, H=H, V=V, N=270, Z=200, zstart=-20, step=0.2, scale=0.1, redundancy=1),
                xfactor=1000.0, name=C2_NAME)


def native_spectrum(spectrum_csv: str, nmat: int = 6):
    """attenuation_coefficient through the product library (mini x-ray DB)."""
    from virtualcbct_b200 import attenuation_table
    return attenuation_table(spectrum_csv, MINIDB, nmat)


def detector_sample_columns(W: int, xshift_px: float = 0.0) -> np.ndarray:
    """Detector columns a sampled parity check covers: both detector edges,
    the central column W/2 (where the reference's two projector twins break
    ties differently) and, for an offset detector, the column under the
    isocentre; eight columns each."""
    cols = set(range(0, 8)) | set(range(W - 8, W)) | set(range(W // 2 - 4, W // 2 + 4))
    if xshift_px:
        c = int(round(W / 2 - xshift_px))
        cols |= set(range(max(0, c - 4), min(W, c + 4)))
    return np.array(sorted(cols), np.int32)


def column_runs(cols: np.ndarray):
    """Consecutive runs [c0, c1) of a sorted column list."""
    runs, start = [], int(cols[0])
    for a, b in zip(cols[:-1], cols[1:]):
        if b != a + 1:
            runs.append((start, int(a) + 1))
            start = int(b)
    runs.append((start, int(cols[-1]) + 1))
    return runs


def native_tables(w: dict):
    """prepareTrigonometricTable of a workload's views through the product
    library (bitwise equal to the reference's own)."""
    from virtualcbct_b200 import trig_tables
    g = w["g"]
    return trig_tables(g.W, g.H, np.deg2rad(w["angles_deg"]), w["xs_proj"], np.zeros(g.V), g.pdet, g.dpn)


def reference_tables(w: dict):
    """The same tables from the reference's own prepareTrigonometricTable
    (oracle/_ref)."""
    import oracle as O
    g = w["g"]
    return O.ref_trig_tables(g.W, g.H, np.deg2rad(w["angles_deg"]), w["xs_proj"], np.zeros(g.V), g.pdet, g.dpn)
