"""The drop-in boundary, end to end on the reference's shipped inputs.

The reference's two programs are built from their unmodified sources by
oracle/Makefile, with libvcbct in place of the GPU projector and of the FDK
filter and backprojection objects:

  oracle/_ref/proj_dropin   Release_CBCT_Projection_CM/main.cpp + its CPU
                            objects, linked against -lvcbct (initializeGPU,
                            reprojectionOnGPU with its "<outputname>.raw"
                            file)
  oracle/_ref/cbct2_dropin  Release_recon_from_forward_pro_float_CM/main.cpp +
                            its loader, linked against -lvcbct
                            (prepareConstMap, filterSinogram,
                            reconstructImage)
  oracle/_ref/cbct2         the reference FDK program, all CPU (the checker)

Each shipped deck (txtfile/IR_waterphantom_36pro.txt and _360pro.txt: the
water-phantom slices with the repeat-last-slice rule, the shipped 101-bin
spectrum; then the matching FDK deck, which reads the projector's output) is
run as the reference runs it, and the written files are compared:
projections with the FP64 oracle on sampled rays of every view and with the
reference's own CPU projector on the fixture's views (1e-5 relative per
pixel); the short volume with the reference's CPU cbct2 on the same
projections (+-1 LSB).  The library's own command-line drivers (vcbct_proj,
vcbct_cbct2) run the same decks and must agree.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O
from measure.workloads import detector_sample_columns
from tests import shipped

pytestmark = pytest.mark.gpu

RTOL = 1e-5
ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
REF = os.path.join(ROOT, "oracle", "_ref")
BIN = os.path.join(ROOT, "virtualcbct_b200", "bin")
GOLD = os.path.join(os.path.dirname(__file__), "golden", "shipped_decks_reference.npz")

DECKS = [("d36", shipped.DECK_36, shipped.FDK_36), ("d360", shipped.DECK_360, shipped.FDK_360)]


def _need(*paths):
    missing = [p for p in paths if not os.path.exists(p)]
    if missing or not shipped.available():
        pytest.skip(f"drop-in builds or staged data missing: {missing or 'oracle/_ref/data'}")


def _run(cmd, cwd, timeout=900):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, f"{cmd[0]} exited {r.returncode}: {r.stderr[-2000:]}"
    return r


def _fdk_deck_fields(rdir, deck):
    cwd = os.getcwd()
    os.chdir(rdir)
    try:
        return O.ref_fdk_load(os.path.join("txtfile", deck))
    finally:
        os.chdir(cwd)


@pytest.mark.parametrize("tag,pdeck,fdeck", DECKS)
def test_reference_programs_run_on_libvcbct(cuda, tmp_path, tag, pdeck, fdeck):
    _need(os.path.join(REF, "proj_dropin"), os.path.join(REF, "cbct2_dropin"), os.path.join(REF, "cbct2"))
    pdir, rdir = shipped.layout(str(tmp_path / "dropin"))
    inp = shipped.projector_inputs(pdir, pdeck)
    g = inp["g"]

    # ---- projector program, unmodified main.cpp on libvcbct
    _run([os.path.join(REF, "proj_dropin"), os.path.join("txtfile", pdeck)], pdir)
    raw = os.path.join(pdir, inp["output_name"] + ".raw")
    out = np.fromfile(raw, np.float32)
    assert out.size == g.V * g.H * g.W
    out = out.reshape(g.V, g.H, g.W)
    assert np.isfinite(out).all() and out.min() > 0.0

    # sampled rays of every view against the FP64 oracle (GPU semantics)
    cols = detector_sample_columns(g.W)
    views = np.arange(g.V) if g.V <= 36 else np.arange(0, g.V, 9)
    og = O.mbfpa_sampled(g, inp["tabs"], inp["vol"], inp["mu"], inp["pdf"], inp["xfactor"], views, cols,
                         want=("d",), exact=False)["d"]
    gpu = out[views][:, :, cols].astype(np.float64)
    rel = np.abs(gpu - og) / og
    shipped.report(f"{tag} drop-in projection vs FP64 oracle (rel/pixel, {len(views)} views x 24 columns)",
                   float(rel.max()))
    assert rel.max() <= RTOL, f"max rel err vs FP64 oracle {rel.max():.3e}"

    # the fixture's views against the reference's own reprojection()
    gold = np.load(GOLD)
    assert int(gold[f"{tag}_volume_checksum"]) == shipped.volume_checksum(inp["vol"])
    assert int(gold[f"{tag}_n_bins"]) == inp["pdf"].shape[0] == 101
    gv, gc = [int(v) for v in gold[f"{tag}_views"]], gold[f"{tag}_cols"]
    args = (g, inp["tabs"], inp["vol"], inp["mu"], inp["pdf"], inp["xfactor"], gv, gc)
    od = O.mbfpa_sampled(*args, want=("d", "f"), exact=False)
    nl = O.mbfpa_sampled(*args, want=("d",), exact=False, with_leng=False)["d"]
    cpu_ties = O.mbfpa_sampled(*args, want=("f",), exact=False, ties=O.TIES_CPU)["f"]
    ref = gold[f"{tag}_out"][:, ::-1, :].astype(np.float64) * (od["d"] / nl)
    gpu = out[gv][:, :, gc].astype(np.float64)
    twin = od["f"] != cpu_ties
    rel = np.abs(gpu - ref) / ref
    shipped.report(f"{tag} drop-in projection vs reprojection() (rel/pixel, 4 views x all 101 bins; tie rays)",
                   [float(rel[~twin].max()), int(twin.sum())])
    assert rel[~twin].max() <= RTOL, f"max rel err vs reprojection() {rel[~twin].max():.3e}"
    assert (np.abs(gpu - od["d"]) / od["d"])[twin].max(initial=0.0) <= RTOL

    # ---- the library's own projector program on the same deck: same file
    cli_p, cli_r = shipped.layout(str(tmp_path / "cli"))
    _run([os.path.join(BIN, "vcbct_proj"), os.path.join("txtfile", pdeck)], cli_p)
    cli_out = np.fromfile(os.path.join(cli_p, inp["output_name"] + ".raw"), np.float32)
    assert np.array_equal(cli_out, out.reshape(-1))

    # ---- FDK program, unmodified main.cpp on libvcbct, reading the file above
    fd = _fdk_deck_fields(rdir, fdeck)
    _run([os.path.join(REF, "cbct2_dropin"), os.path.join("txtfile", fdeck)], rdir)
    vol = np.fromfile(os.path.join(rdir, fd["recon_file"]), np.int16)
    n = fd["recon_size"] ** 2 * fd["recon_slices"]
    assert vol.size == n

    # the reference's CPU cbct2 on the same projections
    ref_p, ref_r = shipped.layout(str(tmp_path / "cpu"))
    shutil.copy(raw, os.path.join(ref_p, os.path.basename(raw)))
    _run([os.path.join(REF, "cbct2"), os.path.join("txtfile", fdeck)], ref_r, timeout=1800)
    ref_vol = np.fromfile(os.path.join(ref_r, fd["recon_file"]), np.int16)
    assert ref_vol.size == n and np.abs(ref_vol).max() > 100
    d = np.abs(vol.astype(np.int32) - ref_vol.astype(np.int32))
    shipped.report(f"{tag} drop-in cbct2 short volume vs the reference cbct2 (LSB, whole volume; voxels off by 1)",
                   [int(d.max()), int((d > 0).sum())])
    assert d.max() <= 1, f"{(d > 1).sum()} voxels differ from the reference cbct2 by more than 1 LSB"

    # the library's own FDK program on the same deck, reading vcbct_proj's file
    _run([os.path.join(BIN, "vcbct_cbct2"), os.path.join("txtfile", fdeck)], cli_r)
    cli_vol = np.fromfile(os.path.join(cli_r, fd["recon_file"]), np.int16)
    d = np.abs(cli_vol.astype(np.int32) - ref_vol.astype(np.int32))
    assert d.max() <= 1
