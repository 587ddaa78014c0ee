"""Full-scale batched forward + adjoint, run as specified: four synthetic
ellipsoid phantoms (seeds 40-43), six FP32 element volumes 512x512x400
(0.5 x 0.5 x 1 mm) each; 720 views of an 800x800 detector (0.5 mm), a 120 kV
spectrum of 111 1-keV bins; 20 gradient iterations of least-squares
material decomposition per phantom (the per-ray spectral state recomputed
from the path integrals kept by each forward launch), then FDK of every
phantom's final projections to 512x512x400 short, with the error of each
output against the FP64 oracle on samples.

Targets are the projections of each phantom with bone P and Ca scaled by
1.1.  Each iteration is one decomposition step (forward + adjoint) at the
current volumes: if its loss is below the last accepted one, the point is
accepted and a step -alpha * grad taken (clamped at zero; alpha starts at
0.5 * loss / |grad|^2 and grows 1.5x after each accepted point); otherwise
the last step is undone and retaken from the accepted point with alpha / 4.
No iteration runs an extra forward.  The whole 80-iteration job is timed
with CUDA events on the launching stream (the per-iteration loss and
gradient norm reads are part of it), after one untimed warm-up step.

    python -m measure.config5          (prints one JSON line)
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

DATA = os.path.join(ROOT, "virtualcbct_b200", "data")
SEEDS = (40, 41, 42, 43)
ITERATIONS = 20


def run(n_iter: int = ITERATIONS, seeds=SEEDS) -> dict:
    import torch

    import oracle as O
    from virtualcbct_b200 import (FILTER_BF16X3, Fdk, FdkGeometry, Projector, ProjGeometry, attenuation_table,
                                  phantoms, trig_tables)
    from virtualcbct_b200.autograd import decomposition_step, project

    g = ProjGeometry(N=512, Z=400, s=0.05, step=0.1, W=800, H=800, V=720)
    ang = np.deg2rad(phantoms.view_angles(g.V))
    tabs = trig_tables(g.W, g.H, ang, np.zeros(g.V), np.zeros(g.V), g.pdet, g.dpn)
    mu, pdf = attenuation_table(os.path.join(DATA, "spectrum_kramers120_111.csv"), os.path.join(DATA, "xraydb_mini"), 6)
    p = Projector(g, *tabs)
    p.set_spectrum(mu, pdf, 1000.0)
    stream = torch.cuda.current_stream()

    vols, targets = [], []
    for seed in seeds:
        truth = phantoms.ellipsoid_phantom_torch(g.N, g.Z, g.s, g.step, seed=seed, as_float=True)
        truth[:, 4:6] *= 1.1
        with torch.no_grad():
            targets.append(project(truth, p).clone())
        del truth
        vols.append(phantoms.ellipsoid_phantom_torch(g.N, g.Z, g.s, g.step, seed=seed, as_float=True))
    nseg = p.count_segments()  # segments of the last loaded volume's geometry (the same rays for all)

    # untimed warm-up on a copy
    w = vols[0].clone()
    decomposition_step(w, targets[0], p)
    del w
    torch.cuda.synchronize()

    losses = [[] for _ in seeds]
    best = [None for _ in seeds]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i, (vol, tgt) in enumerate(zip(vols, targets)):
        acc_vol = torch.empty_like(vol)   # last accepted point and its gradient
        acc_grad = torch.empty_like(vol)
        acc_loss, alpha = None, None
        for _ in range(n_iter):
            loss, grad = decomposition_step(vol, tgt, p)
            lv = float(loss)
            losses[i].append(lv)
            if acc_loss is None or lv < acc_loss:
                acc_loss = lv
                acc_vol.copy_(vol)
                acc_grad.copy_(grad)
                gn = float((grad.double() ** 2).sum())
                alpha = 0.5 * lv / gn if alpha is None else 1.5 * alpha
            else:
                alpha *= 0.25
            del grad
            torch.sub(acc_vol, acc_grad, alpha=alpha, out=vol)
            vol.clamp_(min=0.0)
        best[i] = acc_loss
        vol.copy_(acc_vol)  # the phantom's result: its last accepted point
        del acc_vol, acc_grad
    e1.record(stream)
    torch.cuda.synchronize()
    job_ms = e0.elapsed_time(e1)

    # a plain forward of the same size, for the step / forward ratio
    out = torch.empty_like(targets[0])
    p.load_volume_f32(vols[0])
    p.forward(out)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    p.load_volume_f32(vols[0])
    p.forward(out)
    f1.record(stream)
    torch.cuda.synchronize()
    fwd_ms = f0.elapsed_time(f1)

    # FDK of the projections of every phantom's result
    fg = FdkGeometry(W=800, H=800, V=720, N=512, Z=400, zstart=-20, step=0.1, scale=0.05)
    F = Fdk(fg, ang, np.zeros(fg.V), np.zeros(fg.V))
    fdk_ms, errors = [], {}
    sel = [100, 460]
    for i, vol in enumerate(vols):
        with torch.no_grad():
            proj = project(vol, p).clone()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        filt = F.filter(proj, method=FILTER_BF16X3)
        vf, vi = F.backproject(filt)
        a1.record(stream)
        torch.cuda.synchronize()
        fdk_ms.append(a0.elapsed_time(a1))
        if i == 0:
            # per-output error of phantom 0 against the FP64 oracle on samples
            sub = tuple(np.ascontiguousarray(t[sel]) for t in tabs)
            ref = O.mbfpa_forward(g.with_(V=2), sub, None, mu, pdf, 1000.0, volf=vol.cpu().numpy(),
                                  rows=(384, 416), cols=(300, 316), exact=False, want=("d",))["d"]
            got = proj[sel].cpu().numpy()
            r, c = slice(800 - 416, 800 - 384), slice(300, 316)
            errors["projection_max_rel_vs_fp64"] = float((np.abs(got[:, r, c] - ref[:, r, c]) / ref[:, r, c]).max())
            proj_h = proj.cpu().numpy()
            d64 = O.filter_sinogram(proj_h[sel], np.zeros(2), np.zeros(2), O.fdk_consts(fg.piso), mode=1)
            errors["filter_max_vs_fp64_of_scale"] = float(np.abs(filt[sel].cpu().numpy() - d64).max() / np.abs(d64).max())
            bp64 = O.backproject(fg.N, 2, 0, fg.step, fg.scale, filt.cpu().numpy(), fg.xfactor, ang,
                                 np.zeros(fg.V), O.fdk_consts(fg.piso))
            errors["backprojection_max_vs_fp64_of_scale"] = float(
                np.abs(vf[200:202].cpu().numpy() - bp64).max() / max(1.0, np.abs(bp64).max()))
            errors["short_volume_max_lsb_vs_fp64"] = int(
                np.abs(vi[200:202].cpu().numpy().astype(np.int32) - np.trunc(bp64).astype(np.int32)).max())
        del proj, filt, vf, vi
    steps = len(seeds) * n_iter
    return {"workload": "4 phantoms x 6 FP32 512x512x400 (0.5x0.5x1 mm), 720 views of 800x800 (0.5 mm), "
                        "111 bins; 20 decomposition iterations each, then FDK to 512x512x400 short",
            "iterations": steps, "job_ms": job_ms, "ms_per_iteration": job_ms / steps,
            "forward_ms": fwd_ms, "iteration_over_forward": job_ms / steps / fwd_ms,
            "segments_per_forward": nseg, "loss_first_best": [[l[0], b] for l, b in zip(losses, best)],
            "loss_decreased": all(b < l[0] for l, b in zip(losses, best)),
            "losses_phantom0": losses[0],
            "fdk_ms_per_phantom": fdk_ms, "errors_phantom0": errors}


if __name__ == "__main__":
    print(json.dumps(run()))
