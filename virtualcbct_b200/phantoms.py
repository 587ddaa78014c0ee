"""Seeded synthetic inputs in the reference's formats.

* element volumes: uint16 [Z][6][N][N], element order H, C, N, O, P, Ca, value
  = mass fraction x density [g/cm3] x 1000 (the encoding of the shipped water
  phantoms and of ICRPphantoms_2mmslice/To_material_distribution_for512_random
  .cpp:218-223, which writes percent x density x 10);
* view lists in the flexmap convention ``angle xshift yshift class`` with the
  reference's -0.0001 degree offset (36_little_slide.flexmap:1);
* spectra as ``lo,hi,fraction`` CSV rows in MeV (Spectrum/*.csv).
"""
from __future__ import annotations

import numpy as np

ELEMENTS = ("H", "C", "N", "O", "P", "Ca")

# Mass fractions (H, C, N, O, P, Ca) of the tissue classes; O closes the sum.
TISSUE = {
    "water": (0.111, 0.0, 0.0, 0.889, 0.0, 0.0),
    "soft": (0.102, 0.143, 0.034, 0.719, 0.002, 0.0),
    "lung": (0.103, 0.105, 0.031, 0.759, 0.002, 0.0),
    "bone": (0.034, 0.155, 0.042, 0.441, 0.103, 0.225),
    "fat": (0.114, 0.598, 0.007, 0.281, 0.0, 0.0),
}
DENSITY = {"water": 1.0, "soft": 1.0, "lung": 0.26, "bone": 1.92, "fat": 0.95, "air": 0.0012}


def encode(fractions, density) -> np.ndarray:
    """fraction x density x 1000, rounded to uint16 (per element)."""
    return np.clip(np.rint(np.asarray(fractions, np.float64) * density * 1000.0), 0, 65535).astype(np.uint16)


def water_cylinder(N: int, Z: int, s: float, radius_cm: float, nmat: int = 6) -> np.ndarray:
    """Uniform water cylinder along z (H 111, O 889 inside) in air (N = 1)."""
    c = (np.arange(N) - (N - 1) / 2.0) * s
    r2 = c[None, :] ** 2 + c[:, None] ** 2
    inside = r2 <= radius_cm ** 2
    vol = np.zeros((Z, nmat, N, N), np.uint16)
    w = encode(TISSUE["water"], 1.0)
    for k in range(min(nmat, 6)):
        plane = np.where(inside, w[k], 0).astype(np.uint16)
        if k == 2:
            plane = np.where(inside, plane, 1).astype(np.uint16)  # air: N at 0.0012 g/cm3
        vol[:, k] = plane[None]
    return vol


def random_volume(N: int, Z: int, nmat: int = 6, seed: int = 0, hi: int = 1500) -> np.ndarray:
    """Voxel-wise random element values (a worst case for parity: every voxel
    boundary is a density jump)."""
    rng = np.random.default_rng(seed)
    return rng.integers(0, hi, size=(Z, nmat, N, N)).astype(np.uint16)


def ellipsoid_phantom(N: int, Z: int, s: float, step: float, seed: int = 0,
                      jitter: float = 0.05, as_float: bool = False) -> np.ndarray:
    """Anthropomorphic ellipsoid phantom: body 30 x 22 cm (soft tissue) with a
    fat layer, two lungs (0.26 g/cm3), a spine and a rib ring of cortical bone
    (1.92 g/cm3), in air.  Per-voxel element fractions are jittered by
    +-``jitter`` (relative, uniform) and the oxygen fraction closes the sum,
    as the ICRP conversion does (To_material_distribution_for512_random.cpp:
    151-162).  Returns uint16 codes, or float32 densities x 1000."""
    rng = np.random.default_rng(seed)
    x = (np.arange(N) - (N - 1) / 2.0) * s
    X, Y = np.meshgrid(x, -x)  # row index grows toward -y, as the reference
    zc = (np.arange(Z) - (Z - 1) / 2.0) * step
    cls = np.full((Z, N, N), -1, np.int8)  # -1 air
    names = ["soft", "fat", "lung", "bone"]
    for iz, z in enumerate(zc):
        taper = np.sqrt(max(0.0, 1.0 - (z / (0.5 * Z * step + 20.0)) ** 2))
        body = (X / (15.0 * taper)) ** 2 + (Y / (11.0 * taper)) ** 2 <= 1.0
        inner = (X / (14.0 * taper)) ** 2 + (Y / (10.0 * taper)) ** 2 <= 1.0
        c = np.full((N, N), -1, np.int8)
        c[body] = 1
        c[inner] = 0
        for sx in (-6.0, 6.0):
            lung = ((X - sx) / 4.5) ** 2 + ((Y - 1.0) / 6.5) ** 2 <= 1.0
            c[lung & inner] = 2
        spine = (X / 1.6) ** 2 + ((Y + 7.0) / 1.6) ** 2 <= 1.0
        rr = (X / 12.5) ** 2 + (Y / 8.8) ** 2
        ribs = (rr > 0.93) & (rr < 1.0) & (np.cos(np.arctan2(Y, X) * 9.0 + iz * 0.3) > 0.2)
        c[spine] = 3
        c[ribs & inner] = 3
        cls[iz] = c
    out = np.zeros((Z, 6, N, N), np.float32 if as_float else np.uint16)
    for ci, name in enumerate(names):
        m = cls == ci
        n = int(m.sum())
        if n == 0:
            continue
        base = np.asarray(TISSUE[name], np.float64)
        fr = np.repeat(base[None, :], n, axis=0)
        fr *= 1.0 + rng.uniform(-jitter, jitter, size=fr.shape)
        fr[:, 3] = 1.0 - (fr.sum(axis=1) - fr[:, 3])
        neg = fr[:, 3] < 0
        if neg.any():
            fr[neg] /= fr[neg].sum(axis=1, keepdims=True)
            fr[neg, 3] = 0.0
        rho = DENSITY[name]
        vals = fr * rho * 1000.0
        idx = np.nonzero(m)
        for k in range(6):
            if as_float:
                out[idx[0], k, idx[1], idx[2]] = vals[:, k].astype(np.float32)
            else:
                out[idx[0], k, idx[1], idx[2]] = np.clip(np.rint(vals[:, k]), 0, 65535).astype(np.uint16)
    air = cls < 0
    out[:, 2][air] = 1.2 if as_float else 1
    return out


def view_angles(n_views: int, start_deg: float = -170.0001, span_deg: float = 360.0):
    """Equally spaced view angles (degrees) in the flexmap convention."""
    return start_deg + np.arange(n_views) * (span_deg / n_views)


def flexmap_text(angles_deg, xshift=0.0, yshift=0.0) -> str:
    return "".join(f"{a:.4f} {xshift:g} {yshift:g} 0 \n" for a in angles_deg)


def kramers_spectrum(kvp: float = 100.0, e_lo: float = 10.0, e_hi: float | None = None,
                     width: float = 1.0, mu_filter=None, filter_cm: float = 1.0):
    """Filtered Kramers spectrum in 1 keV bins: fraction proportional to
    (kVp - E)/E * exp(-mu_f(E) t) at the bin midpoints E (keV).  Returns
    (lo_MeV, hi_MeV, fraction) arrays.  ``mu_filter`` maps keV -> 1/cm."""
    e_hi = kvp if e_hi is None else e_hi
    lo = np.arange(e_lo, e_hi, width)
    hi = lo + width
    mid = 0.5 * (lo + hi)
    f = np.clip(kvp - mid, 0.0, None) / mid
    if mu_filter is not None:
        f = f * np.exp(-np.asarray([mu_filter(e) for e in mid]) * filter_cm)
    f = f / f.sum()
    return lo / 1000.0, hi / 1000.0, f


def spectrum_csv_text(lo_mev, hi_mev, frac) -> str:
    rows = ["Energy,1000,Fraction"] + [f"{a:.6g},{b:.6g},{c:.6e}" for a, b, c in zip(lo_mev, hi_mev, frac)]
    return "\n".join(rows) + "\n"


def ellipsoid_phantom_torch(N: int, Z: int, s: float, step: float, seed: int = 0, jitter: float = 0.05,
                            as_float: bool = False, device="cuda"):
    """Same phantom family as ``ellipsoid_phantom``, generated on the GPU with
    a seeded torch generator (for large batched workloads); the element
    encoding and jitter rule are the same, the random stream is not."""
    import torch
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    x = (torch.arange(N, device=device, dtype=torch.float32) - (N - 1) / 2.0) * s
    X = x[None, None, :].expand(Z, N, N)
    Y = (-x)[None, :, None].expand(Z, N, N)
    zc = (torch.arange(Z, device=device, dtype=torch.float32) - (Z - 1) / 2.0) * step
    taper = torch.sqrt(torch.clamp(1.0 - (zc / (0.5 * Z * step + 20.0)) ** 2, min=0.0))[:, None, None]
    cls = torch.full((Z, N, N), -1, dtype=torch.int8, device=device)
    body = (X / (15.0 * taper)) ** 2 + (Y / (11.0 * taper)) ** 2 <= 1.0
    inner = (X / (14.0 * taper)) ** 2 + (Y / (10.0 * taper)) ** 2 <= 1.0
    cls[body] = 1
    cls[inner] = 0
    for sx in (-6.0, 6.0):
        cls[(((X - sx) / 4.5) ** 2 + ((Y - 1.0) / 6.5) ** 2 <= 1.0) & inner] = 2
    rr = (X / 12.5) ** 2 + (Y / 8.8) ** 2
    iz = torch.arange(Z, device=device, dtype=torch.float32)[:, None, None]
    ribs = (rr > 0.93) & (rr < 1.0) & (torch.cos(torch.atan2(Y, X) * 9.0 + iz * 0.3) > 0.2)
    cls[(X / 1.6) ** 2 + ((Y + 7.0) / 1.6) ** 2 <= 1.0] = 3
    cls[ribs & inner] = 3
    names = ["soft", "fat", "lung", "bone"]
    base = torch.zeros((5, 6), device=device, dtype=torch.float32)
    rho = torch.zeros(5, device=device, dtype=torch.float32)
    for ci, name in enumerate(names):
        base[ci] = torch.tensor(TISSUE[name], dtype=torch.float32)
        rho[ci] = DENSITY[name]
    c = cls.long().clamp(min=0)
    fr = base[c]  # [Z,N,N,6]
    fr = fr * (1.0 + (torch.rand(fr.shape, generator=gen, device=device, dtype=torch.float32) * 2 - 1) * jitter)
    fr[..., 3] = 1.0 - (fr.sum(-1) - fr[..., 3])
    neg = fr[..., 3] < 0
    fr[neg] = fr[neg] / fr[neg].sum(-1, keepdim=True)
    fr[..., 3] = torch.where(neg, torch.zeros_like(fr[..., 3]), fr[..., 3])
    vals = fr * rho[c][..., None] * 1000.0
    air = cls < 0
    vals[air] = 0.0
    vals[..., 2] = torch.where(air, torch.full_like(vals[..., 2], 1.2), vals[..., 2])
    vol = vals.permute(0, 3, 1, 2).contiguous()  # [Z][6][N][N]
    if as_float:
        return vol.float()
    return torch.clamp(torch.round(vol), 0, 65535).to(torch.int32).to(torch.int16)  # uint16 bits
