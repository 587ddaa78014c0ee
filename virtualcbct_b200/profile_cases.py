"""Small, self-contained launches of each kernel for profiler captures.

    python -m virtualcbct_b200.profile_cases <case> [repeats]

Each case builds its inputs on the device, runs the kernel ``repeats`` times
(default 2) and prints one line.  The cases are sized to hold a few hundred MB
to a few GB on the device, with inputs larger than the 126 MB L2 where the
kernel streams them, so a profiler capture of one to three launches ends in
seconds:

  forward_c1     MBFPA forward, 20 cm water cylinder 512x512x100 x6 uint16,
                 36 views, 400x400 detector, 90 bins (packed volume 419 MB)
  forward_c2     MBFPA forward of the 25 cm / 512x512x200 / 360-view half-fan
                 workload (packed volume 839 MB; for one-pass launch lists)
  filter_bf16x3  FDK ramp filter, BF16x3 tcgen05 GEMM, 360 views of 400x400
  filter_direct  FDK ramp filter, direct FP32 kernel, same projections
  backproject    FDK backprojection of 360 filtered 400x400 views to 270x270x200
  adjoint_c4     MBFPA adjoint, six float volumes 256x256x64, 90 views, 200x200
  adjoint_state_c4  the same with the forward's path integrals kept
  batch_small    four uneven ellipsoid phantoms (256x256, Z 32-96, V 45-180)
                 in one persistent launch
"""
from __future__ import annotations

import os
import sys

import numpy as np

from . import FILTER_BF16X3, FILTER_DIRECT_F32, Batch, Fdk, FdkGeometry, Projector, ProjGeometry
from . import attenuation_table, phantoms, trig_tables

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
MINIDB = os.path.join(DATA, "xraydb_mini")


def _spectrum(name="spectrum_kramers100_90.csv"):
    return attenuation_table(os.path.join(DATA, name), MINIDB, 6)


def _projector(g, angles_deg, xshift=0.0, spectrum="spectrum_kramers100_90.csv"):
    ang = np.deg2rad(angles_deg)
    tabs = trig_tables(g.W, g.H, ang, np.full(g.V, xshift), np.zeros(g.V), g.pdet, g.dpn)
    p = Projector(g, *tabs)
    mu, pdf = _spectrum(spectrum)
    p.set_spectrum(mu, pdf, 1000.0)
    return p


def _water_forward(N, Z, V, radius, start, xshift):
    import torch
    g = ProjGeometry(N=N, Z=Z, s=0.05, step=0.2, W=400, H=400, V=V)
    p = _projector(g, phantoms.view_angles(V, start), xshift)
    vol = phantoms.water_cylinder(N, Z, g.s, radius)
    p.load_volume(torch.from_numpy(vol.view(np.int16)).cuda())
    return p, torch.empty((V, g.H, g.W), dtype=torch.float32, device="cuda")


def _fdk_inputs():
    import torch
    fg = FdkGeometry(W=400, H=400, V=360, N=270, Z=200, zstart=-20, step=0.2, scale=0.1, redundancy=1)
    ang = np.deg2rad(phantoms.view_angles(360, -180.0001))
    F = Fdk(fg, ang, np.full(360, 16.0), np.zeros(360))
    gen = torch.Generator(device="cuda")
    gen.manual_seed(5)
    proj = 0.05 + torch.rand((fg.V, fg.H, fg.W), generator=gen, device="cuda")
    return F, proj


def run(case: str, repeats: int = 2) -> str:
    import torch
    if case == "forward_c1":
        p, out = _water_forward(512, 100, 36, 10.0, -170.0001, 0.0)
        for _ in range(repeats):
            p.forward(out)
    elif case == "forward_c2":
        p, out = _water_forward(512, 200, 360, 12.5, -180.0001, 1.6)
        for _ in range(repeats):
            p.forward(out)
    elif case in ("filter_bf16x3", "filter_direct"):
        F, proj = _fdk_inputs()
        out = torch.empty_like(proj)
        method = FILTER_BF16X3 if case == "filter_bf16x3" else FILTER_DIRECT_F32
        for _ in range(repeats):
            F.filter(proj, out, method=method)
    elif case == "backproject":
        F, proj = _fdk_inputs()
        filt = F.filter(proj, method=FILTER_DIRECT_F32)
        for _ in range(repeats):
            out = F.backproject(filt)[1]
    elif case == "adjoint_c4":
        g = ProjGeometry(N=256, Z=64, s=0.1, step=0.2, W=200, H=200, V=90)
        p = _projector(g, phantoms.view_angles(90), spectrum="spectrum_kramers100_91.csv")
        vol = phantoms.ellipsoid_phantom_torch(g.N, g.Z, g.s, g.step, seed=21, as_float=True)
        p.load_volume_f32(vol)
        go = torch.ones((g.V, g.H, g.W), dtype=torch.float32, device="cuda")
        out = torch.zeros_like(vol)
        for _ in range(repeats):
            p.adjoint(go, out)
    elif case == "adjoint_state_c4":
        g = ProjGeometry(N=256, Z=64, s=0.1, step=0.2, W=200, H=200, V=90)
        p = _projector(g, phantoms.view_angles(90), spectrum="spectrum_kramers100_91.csv")
        vol = phantoms.ellipsoid_phantom_torch(g.N, g.Z, g.s, g.step, seed=21, as_float=True)
        p.load_volume_f32(vol)
        _, L = p.forward_state()
        go = torch.ones((g.V, g.H, g.W), dtype=torch.float32, device="cuda")
        out = torch.zeros_like(vol)
        for _ in range(repeats):
            p.adjoint_state(L, go, out)
    elif case == "batch_small":
        rng = np.random.default_rng(7)
        b = Batch()
        keep = []
        for i in range(4):
            Z, V = int(rng.integers(32, 97)), int(rng.integers(45, 181))
            g = ProjGeometry(N=256, Z=Z, s=0.125, step=0.4, W=200, H=200, V=V)
            p = _projector(g, phantoms.view_angles(V))
            p.load_volume(phantoms.ellipsoid_phantom_torch(g.N, Z, g.s, g.step, seed=i))
            keep.append(p)
            b.add(p)
        for _ in range(repeats):
            out = b.forward(use_graph=False)[0]
    else:
        raise SystemExit(f"unknown case {case!r}; see the module docstring")
    torch.cuda.synchronize()
    return f"{case}: {repeats} launches ok, checksum {float(out.double().sum()):.6e}"


if __name__ == "__main__":
    print(run(sys.argv[1], int(sys.argv[2]) if len(sys.argv) > 2 else 2))
