"""The reference's shipped inputs (decks, flexmaps, spectrum, x-ray DB,
water-phantom slices) as staged by oracle/Makefile under oracle/_ref/data,
laid out the way the reference's two programs find them: each program runs
in a directory named like its own, the FDK deck reads the projector's output
through ``../Release_CBCT_Projection_CM/``, the projector deck reads the
slices through ``waterphantom/``."""
from __future__ import annotations

import os

import numpy as np

import oracle as O
from measure.workloads import Geometry

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
DATA = os.path.join(ROOT, "oracle", "_ref", "data")
P_NAME = "Release_CBCT_Projection_CM"
R_NAME = "Release_recon_from_forward_pro_float_CM"
DECK_36 = "IR_waterphantom_36pro.txt"
DECK_360 = "IR_waterphantom_360pro.txt"
FDK_36 = "FDK_36pro_water20cm.txt"
FDK_360 = "FDK_360pro_water25cm.txt"


def available() -> bool:
    return os.path.exists(os.path.join(DATA, ".staged"))


def layout(root: str):
    """Create <root>/Release_CBCT_Projection_CM and
    <root>/Release_recon_from_forward_pro_float_CM with links to the staged
    data; returns the two directories."""
    pdir = os.path.join(root, P_NAME)
    rdir = os.path.join(root, R_NAME)
    for d, src in ((pdir, os.path.join(DATA, P_NAME)), (rdir, os.path.join(DATA, R_NAME))):
        os.makedirs(d, exist_ok=True)
        for name in os.listdir(src):
            os.symlink(os.path.join(src, name), os.path.join(d, name))
    os.symlink(os.path.join(DATA, "waterphantom"), os.path.join(pdir, "waterphantom"))
    return pdir, rdir


def projector_inputs(pdir: str, deck: str) -> dict:
    """The projector program's inputs for a shipped deck, built by the
    reference's own code as P/main.cpp builds them: loadData (volume window,
    flexmap), attenuation_coefficient, prepareTrigonometricTable, and
    z_reg = (usedZNumber/2 - zICposition) * z_scale (P/main.cpp:101-103)."""
    cwd = os.getcwd()
    os.chdir(pdir)
    try:
        d = O.ref_proj_load(os.path.join("txtfile", deck))
        mu, pdf = O.ref_attenuation(pdir, d["spectrum"], d["mat_num"], d["mat_type"])
    finally:
        os.chdir(cwd)
    used = d["used_slices"]
    g = Geometry(N=d["recon_size"], Z=used, s=d["x_scale"], step=d["z_scale"], W=d["proj_width"],
                 H=d["proj_height"], V=d["total_proj"], pdet=d["det_pitch_cm"], piso=d["det_pitch_iso_cm"],
                 sad=d["sad_cm"], dpn=d["det_pixel_num"], x_reg=d["x_reg"], y_reg=d["y_reg"],
                 z_reg=(used // 2 - d["z_ic_local"]) * d["z_scale"], nmat=d["mat_num"])
    tabs = O.ref_trig_tables(g.W, g.H, d["angles_rad"], d["xshift"], d["yshift"], g.pdet, g.dpn)
    return dict(g=g, tabs=tabs, vol=d["volume"], mu=mu, pdf=pdf, xfactor=d["xfactor"],
                output_name=d["output_name"], angles_rad=d["angles_rad"], xshift=d["xshift"])


def volume_checksum(vol: np.ndarray) -> int:
    """A cheap fingerprint of a uint16 volume (sum of value x position mod 2^61)."""
    v = vol.reshape(-1).astype(np.uint64)
    idx = np.arange(v.size, dtype=np.uint64) % np.uint64(1000003)
    return int((v * (idx + np.uint64(1))).sum() % np.uint64(2 ** 61 - 1))


def report(key: str, value) -> None:
    """Record a measured error under `key` in the JSON file named by the
    environment variable VCBCT_PARITY_REPORT (no-op when it is unset), so a
    run of the parity tests leaves the numbers behind, not only pass/fail."""
    import json
    path = os.environ.get("VCBCT_PARITY_REPORT")
    if not path:
        return
    data = {}
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
    data[key] = value
    with open(path, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
