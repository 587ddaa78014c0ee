"""Small, self-contained launches of each kernel for profiler captures.

    python -m measure.profile_cases <case> [repeats]

Each case builds its inputs on the device, runs the kernel ``repeats`` times
(default 2) and prints one line.  The cases are sized to hold a few hundred MB
to a few GB on the device, with inputs larger than the 126 MB L2 where the
kernel streams them, so a profiler capture of one to three launches ends in
seconds:

  forward_c1     MBFPA forward, 20 cm water cylinder 512x512x100 x6 uint16,
                 36 views, 400x400 detector, 90 bins (packed volume 839 MB)
  forward_c2     MBFPA forward of the 25 cm / 512x512x200 / 360-view half-fan
                 workload (packed volume 1.68 GB; for one-pass launch lists)
  filter_bf16x3  FDK ramp filter, BF16x3 tcgen05 GEMM, 360 views of 400x400
  filter_direct  FDK ramp filter, direct FP32 kernel, same projections
  backproject    FDK backprojection of 360 filtered 400x400 views to 270x270x200
  adjoint_c4     MBFPA adjoint, six float volumes 256x256x64, 90 views, 200x200
  adjoint_state_c4  the same with the forward's path integrals kept
  batch_small    four uneven ellipsoid phantoms (256x256, Z 32-96, V 45-180)
                 in one persistent launch
  adjoint_state_wide  MBFPA adjoint with kept path integrals, six float
                 volumes 512x512x128 (0.5x0.5x1 mm), 90 views of 800x800,
                 111 bins (the full-scale workload's per-view shape)
  lengthproj_c1  sensitivity backprojection of 36 uint16 400x400 views to
                 512x512x100 (iterative reconstruction)
  ir_update_c1   MLEM/TV update of a 512x512x100 short volume
  noise_c2       reference-unit Gaussian noise on 360 x 400 x 400 floats
  phantom_512    organ numbers -> element values, 512x512x200
"""
from __future__ import annotations

import os
import sys

import numpy as np

from virtualcbct_b200 import FILTER_BF16X3, FILTER_DIRECT_F32, Batch, Fdk, FdkGeometry, Projector, ProjGeometry
from virtualcbct_b200 import attenuation_table, phantoms, trig_tables

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "virtualcbct_b200", "data")
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
    elif case == "adjoint_state_wide":
        g = ProjGeometry(N=512, Z=128, s=0.05, step=0.1, W=800, H=800, V=90)
        p = _projector(g, phantoms.view_angles(90), spectrum="spectrum_kramers120_111.csv")
        vol = phantoms.ellipsoid_phantom_torch(g.N, g.Z, g.s, g.step, seed=40, as_float=True)
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
    elif case in ("lengthproj_c1", "ir_update_c1"):
        from virtualcbct_b200.iterative import ir_update
        g = ProjGeometry(N=512, Z=100, s=0.05, step=0.2, W=400, H=400, V=36)
        p = _projector(g, phantoms.view_angles(g.V))
        gen = torch.Generator(device="cuda")
        gen.manual_seed(3)
        proj = torch.randint(20000, 65000, (g.V, g.H, g.W), generator=gen, device="cuda",
                             dtype=torch.int32).to(torch.int16)
        npf = torch.empty((g.Z, g.N, g.N), dtype=torch.float32, device="cuda")
        p.lengthproj(proj, npf=npf)
        before = torch.randint(0, 3000, (g.Z, g.N, g.N), generator=gen, device="cuda",
                               dtype=torch.int32).to(torch.int16)
        out = npf
        for _ in range(repeats):
            if case == "lengthproj_c1":
                p.lengthproj(proj, npf=npf)
            else:
                out = ir_update(before, npf, npf, g.s, 0.5, 0.002)
    elif case == "noise_c2":
        import ctypes as C

        from virtualcbct_b200 import _native as N
        gen = torch.Generator(device="cuda")
        gen.manual_seed(9)
        out = 5000.0 + 55000.0 * torch.rand(360 * 400 * 400, generator=gen, device="cuda")
        for _ in range(repeats):
            N.check(N.lib().vcbct_gaussian_noise(C.c_void_p(out.data_ptr()), out.numel(), 65535.0, 7, 1, None))
    elif case == "phantom_512":
        import tempfile

        from virtualcbct_b200.icrp import PhantomTables, organs_to_elements
        rng = np.random.default_rng(3)
        with tempfile.TemporaryDirectory() as tmp:
            media, organs = os.path.join(tmp, "m.csv"), os.path.join(tmp, "o.csv")
            with open(media, "w") as f:
                for i in range(1, 53):
                    f.write(",".join([str(i)] + [f"{x:.3f}" for x in rng.uniform(0, 20, 13)]) + "\n")
                f.write("53,0,0,70,30,0,0,0,0,0,0,0,0,0\n")
            with open(organs, "w") as f:
                for k in range(1, 141):
                    f.write(f"{k},{int(rng.integers(1, 53))},{rng.uniform(0.2, 1.9):.3f}\n")
            tabs = PhantomTables(media, organs)
        gen = torch.Generator(device="cuda")
        gen.manual_seed(4)
        ids = torch.randint(0, 141, (200, 512, 512), generator=gen, device="cuda", dtype=torch.int32).to(torch.uint8)
        out = torch.empty((200, 6, 512, 512), dtype=torch.int16, device="cuda")
        for _ in range(repeats):
            organs_to_elements(ids, tabs, out)
    else:
        raise SystemExit(f"unknown case {case!r}; see the module docstring")
    torch.cuda.synchronize()
    return f"{case}: {repeats} launches ok, checksum {float(out.double().sum()):.6e}"


if __name__ == "__main__":
    print(run(sys.argv[1], int(sys.argv[2]) if len(sys.argv) > 2 else 2))
