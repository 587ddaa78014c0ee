"""Generate the spectral data files of virtualcbct_b200/data from the
reference's x-ray database (run where the reference tree is available):

  spectrum_kramers100_90.csv 100 kV filtered Kramers, 1 keV bins 10-100 keV
  spectrum_kramers100_91.csv 100 kV, 91 one-keV bins centred on 10..100 keV
  spectrum_kramers120_111.csv 120 kV, 111 one-keV bins 10-121 keV
  xraydb_mini/{photo,comp,rayl}_5keVto150keV.csv
        the DB rows (same columns: H,C,N,O,P,Ca,energy[eV]) at the bin
        midpoints of these spectra only, so that the attenuation-table
        builder can run without the full 29,001-row tables.

Usage: python virtualcbct_b200/data/make_tables.py [REFERENCE_ROOT]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))
from virtualcbct_b200.phantoms import kramers_spectrum, spectrum_csv_text  # noqa: E402


def main(ref_root):
    P = os.path.join(ref_root, "Release_CBCT_Projection_CM")
    db = {}
    for t in ("photo", "comp", "rayl"):
        path = os.path.join(P, "attenuation_xraydb", f"{t}_5keVto150keV.csv")
        with open(path) as f:
            header = f.readline()
            rows = np.loadtxt(f, delimiter=",")
        db[t] = (header, rows)
    energies_ev = db["photo"][1][:, 6]

    def mu_O_per_cm(e_kev):
        i = int(np.argmin(np.abs(energies_ev - e_kev * 1000.0)))
        return sum(db[t][1][i, 3] for t in ("photo", "comp", "rayl")) * 1.0

    spectra = {}
    with open(os.path.join(P, "Spectrum", "result_20220111_average.csv")) as f:
        shipped = f.read()  # its bin midpoints are added to the mini DB (not copied)
    lo, hi, fr = kramers_spectrum(100.0, 10.0, 100.0, 1.0, mu_O_per_cm, 1.0)
    spectra["spectrum_kramers100_90.csv"] = spectrum_csv_text(lo, hi, fr)
    lo, hi, fr = kramers_spectrum(100.0, 9.5, 100.5, 1.0, mu_O_per_cm, 1.0)
    spectra["spectrum_kramers100_91.csv"] = spectrum_csv_text(lo, hi, fr)
    lo, hi, fr = kramers_spectrum(120.0, 10.0, 121.0, 1.0, mu_O_per_cm, 1.0)
    spectra["spectrum_kramers120_111.csv"] = spectrum_csv_text(lo, hi, fr)

    need = set()
    for name, text in list(spectra.items()) + [(None, shipped)]:
        if name is not None:
            with open(os.path.join(HERE, name), "w") as f:
                f.write(text)
        for line in text.splitlines()[1:]:
            a, b, _ = (float(v) for v in line.split(","))
            mid_ev = float(np.float32(np.float32(a) + np.float32(b))) * 0.5 * 1e6
            need.add(int(np.argmin(np.abs(energies_ev - mid_ev))))
    idx = sorted(need)
    os.makedirs(os.path.join(HERE, "xraydb_mini"), exist_ok=True)
    for t in ("photo", "comp", "rayl"):
        header, rows = db[t]
        with open(os.path.join(HERE, "xraydb_mini", f"{t}_5keVto150keV.csv"), "w") as f:
            f.write(header)
            for i in idx:
                r = rows[i]
                f.write(",".join(repr(float(v)) for v in r[:6]) + f",{int(round(r[6]))}\n")
    print(f"wrote {len(spectra)} spectra and {len(idx)} DB rows")


if __name__ == "__main__":
    # the reference tree: argument, else $VCBCT_REFERENCE, else baseline/_ref
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get(
        "VCBCT_REFERENCE", os.path.join(HERE, "..", "..", "baseline", "_ref"))
    main(ref)
