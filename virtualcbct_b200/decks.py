"""The reference's input decks: the projector's and the FDK's info files
(txt), flexmaps, and the per-slice element volume files.

Readers go through the C library (``vcbct_proj_deck_read``,
``vcbct_fdk_deck_read``, ``vcbct_flexmap_read``,
``vcbct_proj_deck_load_volume``), which follows loadData / loadProjectionData
of Release_CBCT_Projection_CM/projectionData.cpp:63-237 and
Release_recon_from_forward_pro_float_CM/projectionDataMVkV.cpp:51-321.
Writers produce files in the same layout: six header lines, then for every
field a blank line, a comment line and the value line.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N

# Field comments of the projector deck, in file order (projectionData.cpp:78-92).
PROJ_FIELDS = (
    ("spectrum", "X-ray energy spectrum (CSV)"),
    ("total_proj", "total projections"),
    ("proj_width", "projection width"),
    ("proj_height", "projection height"),
    ("angle_file", "angle data file (flexmap)"),
    ("mat_prefix", "element image prefix (slices <prefix>_%03d.raw)"),
    ("z_ic", "isocentre z position (slice number)"),
    ("output_name", "output projection name"),
    ("scale", "voxel pitch x y z [cm]"),
    ("recon_size", "input size (square)"),
    ("recon_slices", "number of slices"),
    ("mat_num", "number of element planes"),
    ("mat_type", "material type"),
    ("xfactor", "density factor"),
    ("reg", "image shift x y z [cm]"),
)

# Field comments of the FDK deck (projectionDataMVkV.cpp:66-92).
FDK_FIELDS = (
    ("energy_class", "X-ray energy label (kV or MV)"),
    ("total_proj", "total projections"),
    ("proj_width", "projection width"),
    ("proj_height", "projection height"),
    ("proj_header_bytes", "projection file header bytes"),
    ("proj_prefix", "projection file (without extension)"),
    ("proj_num_digits", "projection file number digits"),
    ("proj_first_number", "first projection file number (hex for kV)"),
    ("proj_ext", "projection file extension"),
    ("angle_file", "angle data file (flexmap)"),
    ("recon_size", "reconstruction size (square)"),
    ("target_class", "reconstruction target class (* = all)"),
    ("recon_offset", "reconstruction start z [cm] (integer)"),
    ("recon_step", "reconstruction z step [cm]"),
    ("recon_slices", "reconstruction slices"),
    ("recon_scale", "reconstruction voxel size [cm]"),
    ("xfactor", "factor for output CT value"),
    ("recon_file", "reconstructed volume file"),
)

_HEADER = ["/" * 56, "//", "//    VirtualCBCT input deck", "//    keep the header, blank and comment lines",
           "//", "/" * 56]


def _fmt(v) -> str:
    if isinstance(v, (tuple, list, np.ndarray)):
        return " ".join(_fmt(x) for x in v)
    if isinstance(v, float):
        return repr(v)
    return str(v)


def _write_deck(path, fields, values: dict):
    lines = list(_HEADER)
    for name, comment in fields:
        if name not in values:
            raise KeyError(f"deck field {name!r} missing")
        lines += ["", f"// {comment}", _fmt(values[name])]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_proj_deck(path, **values):
    """Write a projector info file.  ``scale`` and ``reg`` are 3-tuples."""
    _write_deck(path, PROJ_FIELDS, values)


def write_fdk_deck(path, **values):
    """Write an FDK info file."""
    _write_deck(path, FDK_FIELDS, values)


def write_flexmap(path, angles_deg, xshift=0.0, yshift=0.0, classes="0"):
    """Flexmap lines ``angle xshift yshift class``."""
    n = len(angles_deg)
    xs = np.broadcast_to(np.asarray(xshift, np.float64), (n,))
    ys = np.broadcast_to(np.asarray(yshift, np.float64), (n,))
    cl = [classes] * n if isinstance(classes, str) else list(classes)
    with open(path, "w") as f:
        for a, x, y, c in zip(angles_deg, xs, ys, cl):
            f.write(f"{a:.5f} {x:g} {y:g} {c} \n")


def _struct_dict(st) -> dict:
    out = {}
    for name, ctype in st._fields_:
        v = getattr(st, name)
        if isinstance(v, bytes):
            v = v.decode()
        elif hasattr(ctype, "_length_"):
            v = np.array(v[:], np.float64)
        out[name] = v
    return out


def read_proj_deck(path) -> dict:
    """Fields of a projector info file plus the derived slice window."""
    d = N.ProjDeckC()
    N.check(N.lib().vcbct_proj_deck_read(str(path).encode(), C.byref(d)))
    out = _struct_dict(d)
    out["_c"] = d
    return out


def load_proj_volume(deck: dict):
    """The deck's element volume, uint16 [used_slices][mat_num][N][N], and
    the number of slice files that were missing or short."""
    d = deck["_c"]
    vol = np.zeros((d.used_slices, d.mat_num, d.recon_size, d.recon_size), np.uint16)
    bad = C.c_int(0)
    N.check(N.lib().vcbct_proj_deck_load_volume(C.byref(d), C.c_void_p(vol.ctypes.data), C.byref(bad)))
    return vol, int(bad.value)


def read_flexmap(path, capacity: int):
    """(angles_rad, xshift, yshift) of the first entries of a flexmap."""
    a, x, y = np.zeros(capacity), np.zeros(capacity), np.zeros(capacity)
    n = C.c_int(0)
    dp = C.POINTER(C.c_double)
    N.check(N.lib().vcbct_flexmap_read(str(path).encode(), int(capacity), a.ctypes.data_as(dp),
                                       x.ctypes.data_as(dp), y.ctypes.data_as(dp), C.byref(n)))
    k = int(n.value)
    return a[:k].copy(), x[:k].copy(), y[:k].copy()


def read_fdk_deck(path) -> dict:
    """Fields of an FDK info file with its filtered (and possibly reversed)
    view list; the per-view arrays are trimmed to total_proj entries."""
    d = N.FdkDeckC()
    N.check(N.lib().vcbct_fdk_deck_read(str(path).encode(), C.byref(d)))
    out = _struct_dict(d)
    for k in ("angles_rad", "xshift", "yshift"):
        out[k] = out[k][: d.total_proj]
    return out
