#!/usr/bin/env python
"""Benchmark of the MBFPA hot path (plus FDK) on synthetic data.

Metric: MBFPA ray-voxel throughput in Gseg/s -- one "segment"
is one in-volume, in-cylinder, non-degenerate segment of the reference's
Siddon-style march that reads one voxel's six element values -- with FDK
backprojection GUPS, the forward+adjoint / forward ratio and the CPU baseline
reported beside it.

Workload (one GPU): "Plain MBFPA + FDK at scale": 25 cm water cylinder,
512x512x200 uint16 x 6 elements (0.5 x 0.5 x 2 mm), 360 views at 1 deg with the
half-fan detector offset (xshift 1.6 in the projector flexmap = 160 px),
400x400 float32 projections, a 100 kV filtered-Kramers spectrum in 1 keV bins
(90 bins); FDK to 270x270x200 (1 mm) with cosine + half-fan weights + ramp.
All inputs are seeded synthetic data in the reference's formats.

A step = one forward projection of the whole stack (every ray, every bin).
`value` is measured with the volume resident in HBM; `e2e` repeats the step
through the C ABI (vcbct_projector_project) with pinned host buffers: volume
upload + re-layout + projection + download inside the timed region, the
upload and download overlapped with the projection by detector row band.

Usage:  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
For N > 1 run under torch.distributed.run: every rank projects its own copy
of the workload (weak scaling, no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DATA = os.path.join(ROOT, "virtualcbct_b200", "data")
MINIDB = os.path.join(DATA, "xraydb_mini")

METRIC = "MBFPA ray-voxel Gseg/s & FDK GUPS; batched vs plain; grad-step/fwd ratio @stated err"

# DRAM traffic of one forward launch of this workload: ncu
# dram__bytes_read.sum + dram__bytes_write.sum of the first launch of
# `python -m measure.profile_cases forward_c2 1` (a one-pass capture
# of the full-size launch): 17.40 GB read + 6.48 GB written.
FORWARD_DRAM_BYTES = 23.88e9


def workload():
    """The C2 workload (measure/workloads.c2_workload) with the product
    library's spectrum table and FDK geometry (the GPU arm)."""
    from measure.workloads import c2_workload, native_spectrum
    w = c2_workload()
    w["mu"], w["pdf"] = native_spectrum(w["spectrum_csv"])
    w["g"] = w["g"].native()
    w["fg"] = w["fdk"].native()
    return w


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) < 9:
                continue
            for n, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def bp_update_counts(fg, ang, xs):
    """Voxel-view updates of a backprojection: all (N^2 Z V, the unit of
    GUPS), inside the circular mask, and effective (inside the mask with the
    projected detector column and row on the detector; the others are
    skipped).  The kernel's geometry restated in float64 (edge cases at the
    detector border may count one either way)."""
    N, Z, V, W, H = fg.N, fg.Z, fg.V, fg.W, fg.H
    R = (N - 1) / 2.0
    y, x = np.mgrid[0:N, 0:N].astype(np.float64)
    m = (y - R) ** 2 + (x - R) ** 2 <= R * R
    cp = N / 2.0 - 0.5
    xx = ((x - cp) * fg.scale)[m]
    yy = (-(y - cp) * fg.scale)[m]
    pitch = fg.piso * fg.mpn / W
    px = fg.pdet * fg.mpn / W
    eff = 0
    for th in range(V):
        cs, sn = np.cos(ang[th]), np.sin(ang[th])
        L2 = 1.0 - (-xx * sn + yy * cs) / fg.sad
        g = 1.0 / (L2 * pitch)
        uu = np.floor((W // 2) + xs[th] / px - 0.5 + (xx * cs + yy * sn) * g)
        ok = (uu >= 0) & (uu <= W - 1)
        gz = g[ok]
        lo = np.ceil((-(H // 2) / gz - fg.zstart) / fg.step)
        hi = np.ceil(((H - H // 2) / gz - fg.zstart) / fg.step)
        eff += int(np.clip(np.minimum(hi, Z) - np.maximum(lo, 0), 0, None).sum())
    return N * N * Z * V, int(m.sum()) * Z * V, eff


def fdk_cpu_baseline(fg, ang, xs, views, proj, filt):
    """The reference's filterSinogram and reconstructImage (compiled from its
    sources, OpenMP on all host cores) on a sample of the views, extrapolated
    linearly in the view count to the whole stack."""
    import oracle as O
    try:
        ncores = os.cpu_count() or 1
        n = len(views)
        _, s_filt = O.ref_filter(proj, xs[views], np.zeros(n), fg.piso, ncores)
        _, s_bp = O.ref_backproject(fg.N, fg.Z, fg.zstart, fg.step, fg.scale, filt, fg.xfactor, ang[views], xs[views],
                                    fg.piso, ncores)
        k = fg.V / n
        bp_s = s_bp * k
        return {"filter_ms": s_filt * k * 1e3, "bp_ms": bp_s * 1e3,
                "bp_gups": fg.N * fg.N * fg.Z * fg.V / bp_s / 1e9, "unit": "ms / GUPS", "cores": ncores,
                "kind": "reference",
                "sample": f"filterSinogram ({s_filt:.2f} s) and reconstructImage ({s_bp:.2f} s) on {n} of "
                          f"{fg.V} views, extrapolated to {fg.V} views"}
    except Exception as e:  # informative, never fatal
        return {"value": None, "kind": "reference", "sample": f"unavailable: {e}"}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_reference_sample(w, tabs, views, bins, nthreads):
    """Time the reference's own CPU projector (oracle/_ref) on (views x bins)."""
    import oracle as O
    with O.quiet_stdout():
        _, secs = O.ref_mbfpa_views(w["g"], tabs, w["vol"], w["mu"], w["pdf"], w["xfactor"], views, bins,
                                    nthreads=nthreads)
    return secs


def segments_per_view_cpu(w, tabs, views):
    """Segment count of the sampled views from the CPU oracle (the unit's
    definition); used by the reference arm, which must not touch the GPU."""
    import oracle as O
    r = O.mbfpa_forward(w["g"], tabs, w["vol"], w["mu"][:, :1], w["pdf"][:1], w["xfactor"],
                        views=views, exact=False, want=("nm",))
    return {int(v): int(r["nm"][v].sum()) for v in views}


def rank_barrier(world):
    """All ranks meet (a no-op for one process)."""
    if world > 1:
        import torch
        torch.distributed.barrier()


def max_over_ranks_on(x, world, device):
    """The largest of every rank's x (each rank's timing); `device` is where
    the process group's backend reduces (a CUDA device for NCCL, "cpu" for
    gloo)."""
    if world > 1:
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())
    return x


def job_rate(units_per_rank, world, ms_max):
    """Whole-job throughput of N replicas: every rank's units over the
    slowest rank's time (in G units per second)."""
    return units_per_rank * world / (ms_max * 1e-3) / 1e9


def run_reference(args, rank, world):
    """Reference arm: the reference's own CPU projector (reprojection(),
    P/reprojection.cpp, compiled from its sources into oracle/_ref) on all
    host threads.  Its inputs are built by the reference's own code too --
    attenuation_coefficient (P/prior_weight_production.cpp:200) on the
    reference's x-ray DB, prepareTrigonometricTable (P/misc.cpp:10) -- and the
    volume by measure/workloads (numpy); segments are counted by the CPU
    oracle.  Nothing of the product library is loaded.

    A step is a bounded sample of the C2 workload: one view per host thread,
    one energy bin.  reprojection() marches every segment once per bin, so
    the rate in the metric's unit (segments of the whole spectral
    projection) is the sample's segments / (its seconds x the bin count);
    ms_per_step is the measured seconds of one sample."""
    if rank != 0:
        return
    import oracle as O
    from measure.workloads import REF_PROJ_DIR, c2_workload, reference_tables
    w = c2_workload()
    g = w["g"]
    if not O.have_reference() or not os.path.isdir(REF_PROJ_DIR):
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref (reference CPU code compiled from its sources) is not built"}))
        return
    w["mu"], w["pdf"] = O.ref_attenuation(REF_PROJ_DIR, w["spectrum_csv"], 6)
    tabs = reference_tables(w)
    ncores = os.cpu_count() or 1
    NE = int(w["pdf"].shape[0])
    nviews = max(1, min(g.V, ncores))
    rng = np.random.default_rng(0)
    seg_cache = {}
    times, segs = [], []
    for it in range(args.warmup + args.steps):
        views = np.sort(rng.choice(g.V, size=nviews, replace=False)).astype(np.int32)
        bins = np.array([rng.integers(NE)], np.int32)
        need = [v for v in views if v not in seg_cache]
        if need:
            seg_cache.update(segments_per_view_cpu(w, tabs, np.array(need, np.int32)))
        t = cpu_reference_sample(w, tabs, views, bins, ncores)
        if it >= args.warmup:
            times.append(t)
            segs.append(sum(seg_cache[int(v)] for v in views) * len(bins))
    per_seg_bin = np.sum(times) / np.sum(segs)       # s per segment per bin
    value = 1.0 / (per_seg_bin * NE) / 1e9           # Gseg/s of the spectral projection
    total_segs = np.mean(list(seg_cache.values())) * g.V
    sample = f"{nviews} views x 1 of {NE} bins per step ({np.mean(times):.2f} s measured per step)"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Gseg/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(times)) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": w["name"], "sample": sample, "parallelism": f"cpu{ncores}"},
        "sample_seconds": [float(t) for t in times],
        "extrapolated_full_step_ms": per_seg_bin * total_segs * NE * 1e3,
        "cpu_baseline": {"value": value, "unit": "Gseg/s", "cores": ncores, "cpu_model": cpu_model(),
                         "kind": "reference",
                         "sample": sample + f"; the full step ({g.V} views x {NE} bins) extrapolates to "
                                           f"{per_seg_bin * total_segs * NE:.0f} s"},
        "e2e": {"value": value, "unit": "Gseg/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def decomposition_section(stream):
    """Config 4: one least-squares decomposition step (forward + adjoint
    through torch.autograd) vs a plain forward: six FP32 element volumes
    256x256x64 (1x1x2 mm), 90 views, 200x200 detector (2 mm), 91-bin 100 kV
    spectrum; target from the same phantom with bone Ca/P +10%."""
    import torch
    from virtualcbct_b200 import Projector, ProjGeometry, attenuation_table, phantoms, trig_tables
    from virtualcbct_b200.autograd import decomposition_step
    g = ProjGeometry(N=256, Z=64, s=0.1, step=0.2, W=200, H=200, V=90)
    ang = np.deg2rad(phantoms.view_angles(g.V))
    tabs = trig_tables(g.W, g.H, ang, np.zeros(g.V), np.zeros(g.V), g.pdet, g.dpn)
    mu, pdf = attenuation_table(os.path.join(DATA, "spectrum_kramers100_91.csv"), MINIDB, 6)
    vol = phantoms.ellipsoid_phantom_torch(g.N, g.Z, g.s, g.step, seed=21, as_float=True)
    tgt_vol = vol.clone()
    tgt_vol[:, 4] *= 1.1
    tgt_vol[:, 5] *= 1.1
    p = Projector(g, *tabs)
    p.set_spectrum(mu, pdf, 1000.0)
    p.load_volume_f32(tgt_vol)
    target = p.forward().clone()
    p.load_volume_f32(vol)
    out = torch.empty_like(target)
    for _ in range(3):
        p.forward(out)
        decomposition_step(vol, target, p)
    torch.cuda.synchronize()
    reps = 5
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e[0].record(stream)
    for _ in range(reps):
        p.load_volume_f32(vol)
        p.forward(out)
    e[1].record(stream)
    for _ in range(reps):
        loss, grad = decomposition_step(vol, target, p)
    e[2].record(stream)
    torch.cuda.synchronize()
    fwd = e[0].elapsed_time(e[1]) / reps
    step = e[1].elapsed_time(e[2]) / reps
    return {"workload": "6 x FP32 256x256x64 (1x1x2 mm), 90 views, 200x200 (2 mm), 91 bins",
            "forward_ms": fwd, "step_ms": step, "step_over_forward": step / fwd,
            "loss": float(loss.item())}


def decomposition_fullscale_section(stream):
    """Config 5 at full size, one of its four phantoms: six FP32 element
    volumes 512x512x400 (0.5x0.5x1 mm), 720 views of 800x800 (0.5 mm), 111-bin
    120 kV spectrum; one decomposition step (the per-ray path integrals, 11 GB,
    kept from the forward launch) and one with them re-marched, vs a plain
    forward; FDK (BF16x3 filter in two column tiles + backprojection) of the
    projections to 512x512x400."""
    import torch
    from virtualcbct_b200 import (FILTER_BF16X3, Fdk, FdkGeometry, Projector, ProjGeometry, attenuation_table,
                                  phantoms, trig_tables)
    from virtualcbct_b200.autograd import decomposition_step
    g = ProjGeometry(N=512, Z=400, s=0.05, step=0.1, W=800, H=800, V=720)
    ang = np.deg2rad(phantoms.view_angles(g.V))
    tabs = trig_tables(g.W, g.H, ang, np.zeros(g.V), np.zeros(g.V), g.pdet, g.dpn)
    mu, pdf = attenuation_table(os.path.join(DATA, "spectrum_kramers120_111.csv"), MINIDB, 6)
    vol = phantoms.ellipsoid_phantom_torch(g.N, g.Z, g.s, g.step, seed=40, as_float=True)
    p = Projector(g, *tabs)
    p.set_spectrum(mu, pdf, 1000.0)
    vol[:, 4:6] *= 1.1
    p.load_volume_f32(vol)
    target = p.forward().clone()
    vol[:, 4:6] /= 1.1
    p.load_volume_f32(vol)
    nseg = p.count_segments()
    out = torch.empty_like(target)
    p.forward(out)
    decomposition_step(vol, target, p)
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e[0].record(stream)
    p.load_volume_f32(vol)
    p.forward(out)
    e[1].record(stream)
    loss, _ = decomposition_step(vol, target, p)
    e[2].record(stream)
    torch.cuda.synchronize()
    fwd, step = e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2])
    r = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    r[0].record(stream)
    decomposition_step(vol, target, p, keep_limit=0)
    r[1].record(stream)
    torch.cuda.synchronize()
    step_rm = r[0].elapsed_time(r[1])
    fg = FdkGeometry(W=800, H=800, V=720, N=512, Z=400, zstart=-20, step=0.1, scale=0.05)
    F = Fdk(fg, ang, np.zeros(fg.V), np.zeros(fg.V))
    filt = F.filter(out, method=FILTER_BF16X3)
    F.backproject(filt)
    torch.cuda.synchronize()
    f = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    f[0].record(stream)
    F.filter(out, filt, method=FILTER_BF16X3)
    f[1].record(stream)
    F.backproject(filt)
    f[2].record(stream)
    torch.cuda.synchronize()
    bp = f[1].elapsed_time(f[2])
    return {"workload": "6 x FP32 512x512x400 (0.5x0.5x1 mm), 720 views, 800x800 (0.5 mm), 111 bins",
            "segments": nseg, "forward_ms": fwd, "forward_gseg_s": nseg / (fwd * 1e-3) / 1e9,
            "step_ms": step, "step_over_forward": step / fwd, "loss": float(loss.item()),
            "step_remarched_ms": step_rm, "step_remarched_over_forward": step_rm / fwd,
            "fdk_filter_ms": f[0].elapsed_time(f[1]), "fdk_bp_ms": bp,
            "fdk_bp_gups": fg.N * fg.N * fg.Z * fg.V / (bp * 1e-3) / 1e9}


def batched_section(stream, args):
    """Config 3: 16 ellipsoid phantoms with uneven slice (64-256) and view
    (90-720) counts, 512x512 slices (0.625 mm), 400x400 detector: one
    persistent launch replayed from a CUDA graph vs one plain launch per
    phantom, both on device-resident volumes."""
    import torch
    from virtualcbct_b200 import Batch, Projector, ProjGeometry, attenuation_table, phantoms, trig_tables
    rng = np.random.default_rng(2024)
    mu, pdf = attenuation_table(os.path.join(DATA, "spectrum_kramers100_90.csv"), MINIDB, 6)
    projs, outs = [], []
    batch = Batch()
    zs, vs = [], []
    for i in range(16):
        Z = int(rng.integers(64, 257))
        V = int(rng.integers(90, 721))
        g = ProjGeometry(N=512, Z=Z, s=0.0625, step=0.2, W=400, H=400, V=V)
        ang = np.deg2rad(phantoms.view_angles(V))
        tabs = trig_tables(g.W, g.H, ang, np.zeros(V), np.zeros(V), g.pdet, g.dpn)
        p = Projector(g, *tabs)
        p.set_spectrum(mu, pdf, 1000.0)
        vol = phantoms.ellipsoid_phantom_torch(g.N, Z, g.s, g.step, seed=100 + i)
        p.load_volume(vol)
        del vol
        projs.append(p)
        outs.append(batch.add(p))
        zs.append(Z)
        vs.append(V)
    torch.cuda.synchronize()
    nseg = sum(p.count_segments() for p in projs)
    tuned = batch.autotune()
    batch.forward(use_graph=True)
    for p, o in zip(projs, outs):
        p.forward(o)
    torch.cuda.synchronize()
    reps = 2
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e[0].record(stream)
    for _ in range(reps):
        for p, o in zip(projs, outs):
            p.forward(o)
    e[1].record(stream)
    for _ in range(reps):
        batch.forward(use_graph=True)
    e[2].record(stream)
    torch.cuda.synchronize()
    plain = e[0].elapsed_time(e[1]) / reps
    bat = e[1].elapsed_time(e[2]) / reps
    return {"workload": "16 ellipsoid phantoms 512x512xZ (Z 64-256), V 90-720, 400x400",
            "slices": zs, "views": vs, "segments": nseg, "autotuned_cols_per_block": tuned, "plain_ms": plain, "batched_graph_ms": bat,
            "batched_over_plain_speedup": plain / bat, "batched_gseg_s": nseg / (bat * 1e-3) / 1e9}


def iterative_section(stream):
    """The projector program's iterative-reconstruction helpers at the
    512x512x100 / 36-view size: sensitivity backprojection of uint16
    projections (lengthproj) and the MLEM/TV update (IR_ImageCBCT)."""
    import torch
    from virtualcbct_b200 import Projector, ProjGeometry, phantoms, trig_tables
    from virtualcbct_b200.iterative import ir_update
    g = ProjGeometry(N=512, Z=100, s=0.05, step=0.2, W=400, H=400, V=36)
    ang = np.deg2rad(phantoms.view_angles(g.V))
    p = Projector(g, *trig_tables(g.W, g.H, ang, np.zeros(g.V), np.zeros(g.V), g.pdet, g.dpn))
    gen = torch.Generator(device="cuda")
    gen.manual_seed(3)
    proj = torch.randint(20000, 65000, (g.V, g.H, g.W), generator=gen, device="cuda", dtype=torch.int32)
    proj = proj.to(torch.int16)  # uint16 bits
    npf = torch.empty((g.Z, g.N, g.N), dtype=torch.float32, device="cuda")
    before = torch.randint(0, 3000, (g.Z, g.N, g.N), generator=gen, device="cuda", dtype=torch.int32).to(torch.int16)
    npf_re = npf.clone()
    out = torch.empty_like(npf)

    def t(f, reps=3):
        f()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            f()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    lp = t(lambda: p.lengthproj(proj, npf=npf))
    npf_re.copy_(npf)
    ir = t(lambda: ir_update(before, npf, npf_re, g.s, 0.5, 0.002, out=out), reps=10)
    nvox = g.N * g.N * g.Z
    peak, peak_kind = measured_peaks()
    ir_bytes = 14.0 * nvox  # short before + float npf, npf_re, out (neighbours from cache)
    res = {"workload": "512x512x100, 36 views of 400x400 uint16",
           "lengthproj_ms": lp, "lengthproj_gvox_views_s": nvox * g.V / (lp * 1e-3) / 1e9,
           "lengthproj_bound": "fp64 (the reference's double arithmetic, about 8 divisions per voxel-view)",
           "ir_update_ms": ir, "ir_update_gvox_s": nvox / (ir * 1e-3) / 1e9,
           "ir_update_roofline": {"bound": "hbm", "achieved": ir_bytes / (ir * 1e-3) / 1e9, "peak": peak,
                                  "unit": "GB/s", "frac": ir_bytes / (ir * 1e-3) / 1e9 / peak,
                                  "peak_kind": peak_kind, "bytes": "14 B per voxel"}}
    try:  # the reference's own lengthproj / IR_ImageCBCT (oracle/_ref), all host threads
        import oracle as O
        if O.have_reference():
            tabs = trig_tables(g.W, g.H, ang, np.zeros(g.V), np.zeros(g.V), g.pdet, g.dpn)
            proj_h = proj.cpu().numpy().view(np.uint16)
            t0 = time.perf_counter()
            O.ref_lengthproj(g, tabs, proj_h, views=(0, 2))
            lp_cpu = (time.perf_counter() - t0) * g.V / 2
            b_h, n_h, r_h = before.cpu().numpy(), npf.cpu().numpy(), npf_re.cpu().numpy()
            t0 = time.perf_counter()
            O.ref_ir_update(g.N, g.Z, g.s, b_h, n_h, r_h, 0.5, 0.002, 0.0)
            ir_cpu = time.perf_counter() - t0
            res["cpu_baseline"] = {"lengthproj_ms": lp_cpu * 1e3, "ir_update_ms": ir_cpu * 1e3,
                                   "cores": os.cpu_count(), "kind": "reference",
                                   "sample": "lengthproj on 2 of 36 views (extrapolated), "
                                             "IR_ImageCBCT on the whole volume"}
    except Exception as e:  # informative, never fatal
        res["cpu_baseline"] = {"sample": f"unavailable: {e}"}
    return res


def noise_section(stream, P, out):
    """Detector noise: the reference-unit kernel (gaussiannoise) over a
    360 x 400 x 400 stack, and the cost of the fused epilogue in the
    projector (forward with noise minus forward without)."""
    import ctypes as C

    import torch
    import virtualcbct_b200 as vc
    n = out.numel()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(9)
    base = 5000.0 + 55000.0 * torch.rand(n, generator=gen, device="cuda")
    y = base.clone()
    lib = vc.lib()

    def ev(f, reps):
        f()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            f()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    sp = C.c_void_p(stream.cuda_stream)
    k_ms = ev(lambda: vc._native.check(lib.vcbct_gaussian_noise(C.c_void_p(y.data_ptr()), n, 65535.0, 7, 1, sp)),
              20)
    plain = ev(lambda: P.forward(out), 3)
    P.set_noise(2.0e5, 65535.0 * 40, seed=3)
    noisy = ev(lambda: P.forward(out), 3)
    P.set_noise(0.0)
    peak, peak_kind = measured_peaks()
    gbs = 8.0 * n / (k_ms * 1e-3) / 1e9
    res = {"workload": "360 x 400 x 400 float projections",
           "kernel_ms": k_ms, "kernel_gpix_s": n / (k_ms * 1e-3) / 1e9,
           "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                        "peak_kind": peak_kind, "bytes": "8 B per pixel (read + write)"},
           "forward_ms": plain, "forward_with_noise_ms": noisy}
    try:
        import oracle as O
        if O.have_reference():
            m = 4_000_000
            h = base[:m].cpu().numpy()
            t0 = time.perf_counter()
            O.ref_gaussiannoise(h, 1)
            secs = time.perf_counter() - t0
            res["cpu_baseline"] = {"value": m / secs / 1e9, "unit": "Gpix/s", "cores": 1, "kind": "reference",
                                   "sample": f"gaussiannoise() on {m} pixels ({secs:.2f} s)"}
    except Exception as e:
        res["cpu_baseline"] = {"sample": f"unavailable: {e}"}
    return res


def phantom_section(stream):
    """Phantom generator: organ numbers -> six element values (the ICRP
    conversion's lookup) over a 512 x 512 x 200 organ volume, with seeded
    synthetic media / organ tables in the reference's CSV formats."""
    import torch
    from virtualcbct_b200.icrp import PhantomTables, organs_to_elements
    tmp = tempfile.mkdtemp(prefix="vcbct_icrp_")
    try:
        rng = np.random.default_rng(3)
        rows = [",".join([str(i)] + [f"{x:.3f}" for x in np.r_[rng.uniform(0, 20, 4), 0, 0,
                                                                  rng.uniform(0, 2, 7)]]) for i in range(1, 53)]
        rows.append("53,0,0,70,30,0,0,0,0,0,0,0,0,0")
        media = os.path.join(tmp, "media.csv")
        organs = os.path.join(tmp, "organs.csv")
        with open(media, "w") as f:
            f.write("\n".join(rows) + "\n")
        with open(organs, "w") as f:
            f.write("\n".join(f"{k},{int(rng.integers(1, 53))},{rng.uniform(0.2, 1.9):.3f}"
                              for k in range(1, 141)) + "\n141,53,0.001\n")
        tabs = PhantomTables(media, organs, seed=1)
        gen = torch.Generator(device="cuda")
        gen.manual_seed(4)
        Z, R = 200, 512
        ids = torch.randint(0, 142, (Z, R, R), generator=gen, device="cuda", dtype=torch.int32).to(torch.uint8)
        out = torch.empty((Z, 6, R, R), dtype=torch.int16, device="cuda")
        organs_to_elements(ids, tabs, out, stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(10):
            organs_to_elements(ids, tabs, out, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 10
        nvox = Z * R * R
        peak, peak_kind = measured_peaks()
        gbs = 13.0 * nvox / (ms * 1e-3) / 1e9
        res = {"workload": "512 x 512 x 200 organ numbers -> 6 x uint16", "ms": ms,
               "gvox_s": nvox / (ms * 1e-3) / 1e9,
               "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                            "peak_kind": peak_kind, "bytes": "13 B per voxel (1 read, 12 written)"}}
        try:
            import oracle as O
            if O.have_icrp_convert():
                ids_h = np.random.default_rng(5).integers(0, 142, size=(100, 271, 543)).astype(np.uint8)
                t0 = time.perf_counter()
                O.ref_icrp_convert(tmp, ids_h, media, organs)
                secs = time.perf_counter() - t0
                res["cpu_baseline"] = {"value": ids_h.size / secs / 1e9, "unit": "Gvox/s", "cores": 1,
                                       "kind": "reference",
                                       "sample": f"the reference converter on its 543x271x100 volume, whole "
                                                 f"program incl. its file I/O ({secs:.2f} s)"}
        except Exception as e:
            res["cpu_baseline"] = {"sample": f"unavailable: {e}"}
        return res
    finally:
        import shutil
        shutil.rmtree(tmp, ignore_errors=True)


def deck_load_section():
    """Input pipeline: a 512x512x100 x 6 uint16 volume as per-slice files of
    a projector deck (315 MB, just written, so mostly in the page cache),
    loaded into the projector by the host reader + one upload, and by the
    streaming loader (pinned slabs, copies and re-layout overlapped)."""
    import shutil
    import time

    import torch
    from virtualcbct_b200 import Projector, ProjGeometry, decks, phantoms, trig_tables
    tmp = tempfile.mkdtemp(prefix="vcbct_deck_")
    cwd = os.getcwd()
    try:
        os.chdir(tmp)
        N, Z, V = 512, 100, 4
        vol = phantoms.water_cylinder(N, Z, 0.05, 10.0)
        for i in range(Z):
            vol[i].tofile(f"elem_{i:03d}.raw")
        decks.write_flexmap("v.flexmap", phantoms.view_angles(V))
        decks.write_proj_deck("p.txt", spectrum="s.csv", total_proj=V, proj_width=64, proj_height=64,
                              angle_file="v.flexmap", mat_prefix="elem", z_ic=50, output_name="o",
                              scale=(0.05, 0.05, 0.2), recon_size=N, recon_slices=Z, mat_num=6, mat_type="human",
                              xfactor=1000.0, reg=(0.0, 0.0, 0.0))
        d = decks.read_proj_deck("p.txt")
        g = ProjGeometry(N=N, Z=d["used_slices"], s=0.05, step=0.2, W=64, H=64, V=V)
        ang = np.deg2rad(phantoms.view_angles(V))
        p = Projector(g, *trig_tables(64, 64, ang, np.zeros(V), np.zeros(V), g.pdet, g.dpn))
        nbytes = d["used_slices"] * 6 * N * N * 2

        def host_path():
            v, _ = decks.load_proj_volume(d)
            p.load_volume(v)
            torch.cuda.synchronize()

        def stream_path():
            p.load_deck(d)

        res = {}
        for name, f in (("host_read_then_upload", host_path), ("streamed_slabs", stream_path)):
            f()
            t0 = time.perf_counter()
            for _ in range(3):
                f()
            dt = (time.perf_counter() - t0) / 3
            res[name + "_ms"] = dt * 1e3
            res[name + "_gb_s"] = nbytes / dt / 1e9
        res["volume_mb"] = nbytes / 1e6
        res["speedup"] = res["host_read_then_upload_ms"] / res["streamed_slabs_ms"]
        return res
    finally:
        os.chdir(cwd)
        shutil.rmtree(tmp, ignore_errors=True)


def batched_small_section(stream, n=64, N=128, zr=(16, 64), vr=(18, 90), det=64, s=0.25, step=0.5, seed=77):
    """Many small phantoms (default: 64 of 128x128xZ, Z 16-64, V 18-90, 64x64
    detector; `bench.py` also runs 256 tiny ones: 64x64xZ, Z 8-24, V 8-24,
    32x32): the regime where one launch per phantom leaves the GPU idle
    between launches.  Plain = one projector launch per phantom issued from
    the host (a Python loop, as a user would write it); batched = the
    autotuned batch replayed from its CUDA graph, and the persistent and
    flat single-launch strategies forced."""
    import torch
    from virtualcbct_b200 import Batch, Projector, ProjGeometry, attenuation_table, phantoms, trig_tables
    rng = np.random.default_rng(seed)
    mu, pdf = attenuation_table(os.path.join(DATA, "spectrum_kramers100_90.csv"), MINIDB, 6)
    projs, outs = [], []
    for i in range(n):
        Z = int(rng.integers(zr[0], zr[1] + 1))
        V = int(rng.integers(vr[0], vr[1] + 1))
        g = ProjGeometry(N=N, Z=Z, s=s, step=step, W=det, H=det, V=V)
        ang = np.deg2rad(phantoms.view_angles(V))
        tabs = trig_tables(g.W, g.H, ang, np.zeros(V), np.zeros(V), g.pdet, g.dpn)
        p = Projector(g, *tabs)
        p.set_spectrum(mu, pdf, 1000.0)
        p.load_volume(phantoms.ellipsoid_phantom_torch(g.N, Z, g.s, g.step, seed=500 + i))
        projs.append(p)
    nseg = sum(p.count_segments() for p in projs)
    b_auto, b_pers, b_flat = Batch(), Batch(), Batch()
    for p in projs:
        outs.append(b_auto.add(p))
        b_pers.add(p)
        b_flat.add(p)
    b_pers.configure(Batch.PERSISTENT, 4)
    b_flat.configure(Batch.FLAT, 4)
    tuned = b_auto.autotune()

    def t(f, reps=5):
        f()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            f()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    plain = t(lambda: [p.forward(o) for p, o in zip(projs, outs)])
    auto = t(lambda: b_auto.forward(use_graph=True))
    pers = t(lambda: b_pers.forward(use_graph=True))
    flat = t(lambda: b_flat.forward(use_graph=True))
    return {"workload": f"{n} ellipsoid phantoms {N}x{N}xZ (Z {zr[0]}-{zr[1]}), V {vr[0]}-{vr[1]}, {det}x{det}",
            "segments": nseg, "autotuned": tuned, "plain_ms": plain, "batched_graph_ms": auto,
            "persistent_graph_ms": pers, "flat_graph_ms": flat, "batched_over_plain_speedup": plain / auto,
            "persistent_over_plain_speedup": plain / pers, "flat_over_plain_speedup": plain / flat}


def run_ours(args, rank, world, local_rank):
    import torch
    import virtualcbct_b200 as vc
    from virtualcbct_b200 import Fdk, Projector, trig_tables

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    w = workload()
    g = w["g"]
    ang = np.deg2rad(w["angles_deg"])
    tabs = trig_tables(g.W, g.H, ang, w["xs_proj"], np.zeros(g.V), g.pdet, g.dpn)
    P = Projector(g, *tabs)
    P.set_spectrum(w["mu"], w["pdf"], w["xfactor"])
    vol_h = torch.from_numpy(w["vol"].view(np.int16)).pin_memory()
    vol_d = vol_h.to(dev)
    P.load_volume(vol_d)
    out = torch.empty((g.V, g.H, g.W), dtype=torch.float32, device=dev)
    nseg = P.count_segments()
    stream = torch.cuda.current_stream()

    def barrier():
        rank_barrier(world)

    def max_over_ranks(x):
        return max_over_ranks_on(x, world, dev)

    # ---- device-resident step
    for _ in range(max(3, args.warmup)):
        P.forward(out)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        P.forward(out)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    value = job_rate(nseg, world, ms)

    # ---- end-to-end through the C ABI with pinned host buffers
    out_h = torch.empty((g.V, g.H, g.W), dtype=torch.float32).pin_memory()
    out_np = out_h.numpy()
    vol_np = vol_h.numpy().view(np.uint16)
    lib = vc.lib()
    import ctypes as C
    h = P._h
    sp = C.c_void_p(stream.cuda_stream)

    def e2e_step():  # host volume in, host projections out: one reprojectionOnGPU call's work
        vc._native.check(lib.vcbct_projector_project(h, C.c_void_p(vol_np.ctypes.data),
                                                     C.c_void_p(out_np.ctypes.data), sp))

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    barrier()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    t1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(t0.elapsed_time(t1) / args.steps)
    e2e = job_rate(nseg, world, ms_e2e)
    P.load_volume(vol_d)

    # ---- FDK on the projections just made (device resident)
    fg = w["fg"]
    F = Fdk(fg, ang, w["xs_fdk"], np.zeros(fg.V))
    P.forward(out)
    filt_d = F.filter(out, method=vc.FILTER_DIRECT_F32)
    filt = F.filter(out, method=vc.FILTER_BF16X3)
    filt_err = float((filt - filt_d).abs().max() / filt_d.abs().max())
    vf, vi = F.backproject(filt)
    for _ in range(2):
        F.filter(out, filt_d, method=vc.FILTER_DIRECT_F32)
        F.filter(out, filt, method=vc.FILTER_BF16X3)
        F.backproject(filt)
    torch.cuda.synchronize()
    a0, a1, a2, a3 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
    a0.record(stream)
    for _ in range(args.steps):
        F.filter(out, filt_d, method=vc.FILTER_DIRECT_F32)
    a1.record(stream)
    for _ in range(args.steps):
        F.filter(out, filt, method=vc.FILTER_BF16X3)
    a2.record(stream)
    for _ in range(args.steps):
        F.backproject(filt)
    a3.record(stream)
    torch.cuda.synchronize()
    ms_filter_direct = a0.elapsed_time(a1) / args.steps
    ms_filter = a1.elapsed_time(a2) / args.steps
    ms_bp = a2.elapsed_time(a3) / args.steps
    gups = fg.N * fg.N * fg.Z * fg.V / (ms_bp * 1e-3) / 1e9
    n_all, n_mask, n_eff = bp_update_counts(fg, ang, w["xs_fdk"])
    # BF16x3 work: 6 split products of a (V*H) x Kp x Np GEMM
    Kp = (fg.W + 63) // 64 * 64
    Np = (fg.W + 15) // 16 * 16
    gemm_tflops = 2.0 * 6 * fg.V * fg.H * Kp * Np / (ms_filter * 1e-3) / 1e12
    # host copies of a view sample for the reference FDK's CPU timing
    fdk_views = np.arange(0, fg.V, 10)
    fdk_proj_h = out[torch.from_numpy(fdk_views).to(dev)].cpu().numpy()
    fdk_filt_h = filt[torch.from_numpy(fdk_views).to(dev)].cpu().numpy()
    del F, filt_d

    extra = {}
    if not args.no_extras:
        extra["decomposition"] = decomposition_section(stream)
        extra["decomposition_fullscale"] = decomposition_fullscale_section(stream)
        extra["batched"] = batched_section(stream, args)
        extra["batched_small"] = batched_small_section(stream)
        extra["batched_tiny"] = batched_small_section(stream, n=256, N=64, zr=(8, 24), vr=(8, 24), det=32, s=0.4,
                                                      step=0.8, seed=78)
        extra["iterative"] = iterative_section(stream)
        extra["deck_load"] = deck_load_section()
        extra["noise"] = noise_section(stream, P, out)
        extra["phantom"] = phantom_section(stream)

    # measured gather rooflines: the projector's and the backprojector's
    # access patterns replayed without arithmetic on this device
    from measure import probe_gather
    probe_fwd = probe_gather(3) / 1e9
    probe_fwd_u16 = probe_gather(0) / 1e9
    probe_bp_smem = probe_gather(1) / 1e9
    probe_bp_l1 = probe_gather(2) / 1e9
    gather_roof = {
        "mbfpa": {"pattern": "ray-front 32-B float record gather (11-record runs, stride Z), "
                             "the records the projector reads",
                  "peak_gseg_s": probe_fwd, "achieved_gseg_s": value, "frac": value / probe_fwd,
                  "peak_gseg_s_16b_records": probe_fwd_u16, "frac_16b_records": value / probe_fwd_u16},
        "bp": {"pattern": "bilinear detector-tile gather", "peak_gups_shared": probe_bp_smem,
               "peak_gups_l1": probe_bp_l1,
               "achieved_gups": n_eff / (ms_bp * 1e-3) / 1e9,
               "frac": n_eff / (ms_bp * 1e-3) / 1e9 / max(probe_bp_smem, probe_bp_l1),
               "achieved_gups_all_grid": gups,
               "frac_all_grid": gups / max(probe_bp_smem, probe_bp_l1),
               "note": "achieved_gups counts the effective voxel-view updates (inside the mask, "
                       "detector column and row present: the four taps gathered), "
                       f"{n_eff / n_all:.3f} of the grid's N^2 Z V here (half-fan offset, 40 cm slab "
                       "against the cone); the all-grid rate is the GUPS of the fdk section"},
    }

    peak, peak_kind = measured_peaks()
    alg_bytes = 12.0 * nseg
    achieved = alg_bytes / (ms * 1e-3) / 1e9
    res = {
        "metric": METRIC, "value": value, "unit": "Gseg/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": w["name"], "segments_per_step": nseg, "parallelism": f"replica{world}",
                   "l2": "inputs larger than L2 (packed volume 1.68 GB)"},
        "e2e": {"value": e2e, "unit": "Gseg/s", "ms_per_step": ms_e2e,
                "h2d_bytes_per_step": int(vol_np.nbytes), "d2h_bytes_per_step": int(out_np.nbytes)},
        "gpu_launches": args.steps * 1,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": FORWARD_DRAM_BYTES,
                     "note": "achieved = 12 B (6 x uint16) per segment / forward launch time"},
        "fdk": {"filter_ms": ms_filter, "filter_method": "bf16x3_tcgen05", "filter_tflops": gemm_tflops,
                "filter_ms_direct_f32": ms_filter_direct, "bf16x3_vs_direct_max_rel": filt_err,
                "bp_ms": ms_bp, "bp_gups": gups,
                "bp_gups_in_mask": n_mask / (ms_bp * 1e-3) / 1e9,
                "bp_gups_effective": n_eff / (ms_bp * 1e-3) / 1e9,
                "bp_updates": {"all": n_all, "in_mask": n_mask, "effective": n_eff},
                "short_volume_range": [int(vi.min().item()), int(vi.max().item())]},
        "clocks": clk,
        "gather_roof": gather_roof,
    }
    res.update(extra)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            ncores = os.cpu_count() or 1
            nviews = max(1, min(g.V, ncores))
            views = np.arange(0, g.V, max(1, g.V // nviews))[:nviews].astype(np.int32)
            bins = np.array([w["pdf"].shape[0] // 2], np.int32)
            secs = cpu_reference_sample(w, tabs, views, bins, ncores)
            per_view = nseg / g.V
            full = secs * (g.V / len(views)) * w["pdf"].shape[0]
            res["cpu_baseline"] = {"value": nseg / full / 1e9, "unit": "Gseg/s", "cores": ncores,
                                   "cpu_model": cpu_model(), "kind": "reference",
                                   "sample": f"reprojection() on {len(views)} views x 1 of "
                                             f"{w['pdf'].shape[0]} bins ({secs:.1f} s), "
                                             f"extrapolated to {g.V} views x all bins",
                                   "segments_per_view": per_view}
        except Exception as e:  # the baseline is informative, never fatal
            res["cpu_baseline"] = {"value": None, "unit": "Gseg/s", "cores": os.cpu_count(),
                                   "kind": "reference", "sample": f"unavailable: {e}"}
        res["fdk"]["cpu_baseline"] = fdk_cpu_baseline(fg, ang, w["xs_fdk"], fdk_views, fdk_proj_h, fdk_filt_h)
    if rank == 0:
        print(json.dumps(res))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the decomposition-step and batched sections")
    ap.add_argument("--config5", action="store_true",
                    help="run only the full-scale batched forward + adjoint workload as specified (4 phantoms x "
                         "20 iterations, then FDK; several minutes) and print its JSON line")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.config5:
        if rank == 0:
            from measure.config5 import run as run_config5
            print(json.dumps({"config5": run_config5()}))
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
