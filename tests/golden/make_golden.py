"""Generate the golden fixtures of tests/golden from the reference's own CPU
code (oracle/_ref, compiled from the reference sources by oracle/Makefile).
Run where the reference tree exists:  python tests/golden/make_golden.py

  attenuation.npz  attenuation_coefficient() outputs (mu [6][NE], pdf [NE]) for
                   the shipped 100 kV spectrum and the synthetic Kramers one
  mbfpa_small.npz  reprojection() (CPU twin, per view and bin, float-summed
                   over bins) of a seeded random volume; inputs are regenerated
                   from the stored seed and geometry
  fdk_small.npz    filterSinogram() and reconstructImage() of seeded
                   projections
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from oracle.refpath import reference_root  # noqa: E402
from tests.cases import proj_case  # noqa: E402
from tests.test_fdk_gpu import _case as fdk_case  # noqa: E402

REF = sys.argv[1] if len(sys.argv) > 1 else reference_root()
P = os.path.join(REF, "Release_CBCT_Projection_CM")


def main():
    if not O.have_reference():
        raise SystemExit("build oracle/_ref first (make -C oracle)")
    mu_s, pdf_s = O.ref_attenuation(P, os.path.join(P, "Spectrum", "result_20220111_average.csv"), 6)
    mu_k, pdf_k = O.ref_attenuation(P, os.path.join(ROOT, "virtualcbct_b200", "data",
                                                   "spectrum_kramers100_90.csv"), 6)
    np.savez_compressed(os.path.join(HERE, "attenuation.npz"), mu_shipped=mu_s, pdf_shipped=pdf_s,
                        mu_kramers=mu_k, pdf_kramers=pdf_k)

    g, tabs, vol, ang = proj_case("random", seed=11, hi=600)
    bins = np.arange(pdf_s.shape[0])
    out, _ = O.ref_mbfpa_views(g, tabs, vol, mu_s, pdf_s, 1000.0, np.arange(g.V), bins)
    np.savez_compressed(os.path.join(HERE, "mbfpa_small.npz"), out=out, seed=11, hi=600,
                        angles=ang, cos=tabs[0], sin=tabs[1], xc=tabs[2], yc=tabs[3])

    fg, proj, fang, xs = fdk_case(V=8, seed=5, xshift=1.0)
    filt, _ = O.ref_filter(proj, xs, np.zeros(fg.V), fg.piso)
    vol_d, _ = O.ref_backproject(fg.N, fg.Z, fg.zstart, fg.step, fg.scale, filt, fg.xfactor, fang,
                                 xs, fg.piso)
    np.savez_compressed(os.path.join(HERE, "fdk_small.npz"), proj=proj, filt=filt, vol=vol_d,
                        angles=fang, xshift=xs)
    print("golden fixtures written")


if __name__ == "__main__":
    main()
