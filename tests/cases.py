"""Shared, seeded test cases (small enough for the CPU oracle)."""
from __future__ import annotations

import os

import numpy as np

from virtualcbct_b200 import ProjGeometry, attenuation_table, trig_tables
from virtualcbct_b200 import phantoms

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
DATA = os.path.join(ROOT, "virtualcbct_b200", "data")
MINIDB = os.path.join(DATA, "xraydb_mini")


def spectrum(name="spectrum_kramers100_90.csv", nmat=6):
    return attenuation_table(os.path.join(DATA, name), MINIDB, nmat)


def proj_case(kind="random", N=64, Z=16, s=0.2, step=0.5, W=48, H=40, V=4, dpn=480.0,
              z_reg=0.3, seed=0, angles=None, xshift=0.0, hi=300):
    """Geometry, view tables and element volume of a small projection case."""
    g = ProjGeometry(N=N, Z=Z, s=s, step=step, W=W, H=H, V=V, dpn=dpn, z_reg=z_reg)
    if angles is None:
        angles = phantoms.view_angles(V)
    ang = np.deg2rad(np.asarray(angles, np.float64))
    xs = np.full(V, xshift, np.float64)
    tabs = trig_tables(W, H, ang, xs, np.zeros(V), g.pdet, g.dpn)
    if kind == "random":
        vol = phantoms.random_volume(N, Z, seed=seed, hi=hi)
    elif kind == "water":
        vol = phantoms.water_cylinder(N, Z, s, 0.4 * N * s)
    elif kind == "ellipsoid":
        vol = phantoms.ellipsoid_phantom(N, Z, s, step, seed=seed)
    else:
        raise ValueError(kind)
    return g, tabs, vol, ang
