"""Generate the at-scale golden fixtures from the reference's own CPU
projector (reprojection(), P/reprojection.cpp, compiled from its sources into
oracle/_ref by oracle/Makefile).  Run where the reference tree was staged
(make -C oracle):  python tests/golden/make_golden_scale.py

reprojection() marches one view for one energy bin per call (its view loop
is fixed to view 0, P/reprojection.cpp:45); the fixtures hold, for a few
views, the float sum over every bin in bin order (as P/main.cpp's CPU loop
sums them, :144-148) on the sampled detector columns of every row, in the
reference's CPU-twin layout (no cos^3 factor, rows not flipped).

  c2_reference_sample.npz     the 25 cm / 512x512x200 / 360-view half-fan
                              workload of measure/workloads.c2_workload,
                              4 views x 90 bins
  shipped_decks_reference.npz the reference's shipped decks
                              (txtfile/IR_waterphantom_36pro.txt and
                              IR_waterphantom_360pro.txt: water-phantom slices
                              with the repeat-last-slice rule, the shipped
                              101-bin spectrum), 4 views x 101 bins each
"""
import os
import shutil
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from measure.workloads import c2_workload, detector_sample_columns, native_spectrum, reference_tables  # noqa: E402
from tests import shipped  # noqa: E402

C2_VIEWS = [0, 90, 181, 270]
D36_VIEWS = [0, 9, 18, 27]
D360_VIEWS = [0, 90, 180, 270]


def sample(g, tabs, vol, mu, pdf, xf, views, cols):
    bins = np.arange(pdf.shape[0], dtype=np.int32)
    out, secs = O.ref_mbfpa_views(g, tabs, vol, mu, pdf, xf, np.array(views, np.int32), bins)
    return out[views][:, :, cols].copy(), secs


def main():
    if not (O.have_reference() and shipped.available()):
        raise SystemExit("build oracle/_ref first (make -C oracle)")
    w = c2_workload()
    g = w["g"]
    mu, pdf = native_spectrum(w["spectrum_csv"])
    cols = detector_sample_columns(g.W, 160)
    t0 = time.time()
    out, _ = sample(g, reference_tables(w), w["vol"], mu, pdf, w["xfactor"], C2_VIEWS, cols)
    np.savez_compressed(os.path.join(HERE, "c2_reference_sample.npz"), views=np.array(C2_VIEWS), cols=cols,
                        out=out, volume_checksum=shipped.volume_checksum(w["vol"]))
    print(f"c2 sample: {time.time() - t0:.0f} s")

    tmp = tempfile.mkdtemp(prefix="vcbct_golden_")
    try:
        pdir, _ = shipped.layout(tmp)
        res = {}
        for tag, deck, views in (("d36", shipped.DECK_36, D36_VIEWS), ("d360", shipped.DECK_360, D360_VIEWS)):
            t0 = time.time()
            d = shipped.projector_inputs(pdir, deck)
            dcols = detector_sample_columns(d["g"].W)
            out, _ = sample(d["g"], d["tabs"], d["vol"], d["mu"], d["pdf"], d["xfactor"], views, dcols)
            res.update({f"{tag}_views": np.array(views), f"{tag}_cols": dcols, f"{tag}_out": out,
                        f"{tag}_volume_checksum": shipped.volume_checksum(d["vol"]),
                        f"{tag}_n_bins": d["pdf"].shape[0]})
            print(f"{deck}: {time.time() - t0:.0f} s")
        np.savez_compressed(os.path.join(HERE, "shipped_decks_reference.npz"), **res)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    print("at-scale golden fixtures written")


if __name__ == "__main__":
    main()
