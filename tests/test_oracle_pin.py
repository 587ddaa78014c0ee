"""Pin the CPU oracle (test infrastructure) to the reference.

The golden fixtures are outputs of the reference's own CPU code compiled from
its sources (tests/golden/make_golden.py); the restated oracle must reproduce
them bitwise.  Where the reference objects are built (oracle/_ref), larger
cases are also compared live."""
import os

import numpy as np
import pytest

import oracle as O
from oracle.refpath import reference_path
from tests.cases import DATA, MINIDB, proj_case
from virtualcbct_b200 import attenuation_table

GOLD = os.path.join(os.path.dirname(__file__), "golden")
REF_P = reference_path("Release_CBCT_Projection_CM")


def test_attenuation_builder_matches_reference_golden():
    gold = np.load(os.path.join(GOLD, "attenuation.npz"))
    mu, pdf = attenuation_table(os.path.join(DATA, "spectrum_kramers100_90.csv"), MINIDB, 6)
    assert np.array_equal(mu, gold["mu_kramers"]) and np.array_equal(pdf, gold["pdf_kramers"])


@pytest.mark.skipif(not os.path.isdir(REF_P), reason="reference tree not present")
def test_attenuation_builder_matches_reference_live():
    spec = os.path.join(REF_P, "Spectrum", "result_20220111_average.csv")
    mu, pdf = attenuation_table(spec, os.path.join(REF_P, "attenuation_xraydb"), 6)
    gold = np.load(os.path.join(GOLD, "attenuation.npz"))
    assert np.array_equal(mu, gold["mu_shipped"]) and np.array_equal(pdf, gold["pdf_shipped"])
    mu2, pdf2 = attenuation_table(spec, MINIDB, 6)
    assert np.array_equal(mu2, mu) and np.array_equal(pdf2, pdf)


def test_mbfpa_oracle_reproduces_reference_golden():
    gold = np.load(os.path.join(GOLD, "mbfpa_small.npz"))
    att = np.load(os.path.join(GOLD, "attenuation.npz"))
    g, tabs, vol, _ = proj_case("random", seed=int(gold["seed"]), hi=int(gold["hi"]))
    for a, b in zip(tabs, (gold["cos"], gold["sin"], gold["xc"], gold["yc"])):
        assert np.array_equal(a, b)
    o = O.mbfpa_forward(g, tabs, vol, att["mu_shipped"], att["pdf_shipped"], 1000.0,
                        ties=O.TIES_CPU, with_leng=False, flip=False, exact=True, want=("f",))
    assert np.array_equal(o["f"], gold["out"])


@pytest.mark.skipif(not O.have_reference(), reason="reference objects not built")
@pytest.mark.parametrize("kind,seed", [("water", 0), ("ellipsoid", 2), ("random", 4)])
def test_mbfpa_oracle_reproduces_reference_live(kind, seed):
    g, tabs, vol, _ = proj_case(kind, seed=seed, V=3)
    att = np.load(os.path.join(GOLD, "attenuation.npz"))
    mu, pdf = att["mu_kramers"], att["pdf_kramers"]
    bins = np.arange(0, pdf.shape[0], 7)
    ref, _ = O.ref_mbfpa_views(g, tabs, vol, mu, pdf, 1000.0, np.arange(g.V), bins)
    # restrict the oracle to the same bins: zero the other pdf entries is not
    # equivalent (float sums), so compare bin by bin summed in the same order
    sub_mu = np.ascontiguousarray(mu[:, bins])
    sub_pdf = np.ascontiguousarray(pdf[bins])
    o = O.mbfpa_forward(g, tabs, vol, sub_mu, sub_pdf, 1000.0, ties=O.TIES_CPU, with_leng=False,
                        flip=False, exact=True, want=("f",))
    assert np.array_equal(o["f"], ref)


def test_fdk_oracle_reproduces_reference_golden():
    gold = np.load(os.path.join(GOLD, "fdk_small.npz"))
    proj, xs, ang = gold["proj"], gold["xshift"], gold["angles"]
    V, H, W = proj.shape
    c = O.fdk_consts(0.032509752)
    filt = O.filter_sinogram(proj, xs, np.zeros(V), c, mode=0)
    assert np.array_equal(filt, gold["filt"])
    vol = O.backproject(27, 8, -3, 0.5, 0.4, gold["filt"], 1000, ang, xs, c)
    assert np.array_equal(vol, gold["vol"])


@pytest.mark.skipif(not O.have_reference(), reason="reference objects not built")
def test_const_map_and_mask_match_reference():
    for W in (48, 400):
        assert np.array_equal(O.const_map(W, O.fdk_consts(0.032509752)), O.ref_const_map(W, 0.032509752))
    for N in (27, 270):
        assert np.array_equal(O.mask(N), O.ref_mask(N))


def test_oracle_gpu_and_cpu_twins_differ_only_on_tie_rays():
    """The two reference twins differ only by their tie rules: on the central
    detector column (rays through the rotation axis, y = 0 exactly).  That
    column is H/2: the projector's column shift uses the detector height
    (misc.cpp:31)."""
    g, tabs, vol, _ = proj_case("random", seed=3)
    att = np.load(os.path.join(GOLD, "attenuation.npz"))
    mu, pdf = att["mu_kramers"], att["pdf_kramers"]
    a = O.mbfpa_forward(g, tabs, vol, mu, pdf, 1000.0, ties=O.TIES_GPU, want=("f",))["f"]
    b = O.mbfpa_forward(g, tabs, vol, mu, pdf, 1000.0, ties=O.TIES_CPU, want=("f",))["f"]
    cols = np.unique(np.nonzero(a != b)[2])
    assert set(cols.tolist()) <= {g.H // 2}


GOLD_C2 = os.path.join(GOLD, "c2_reference_sample.npz")
GOLD_DECKS = os.path.join(GOLD, "shipped_decks_reference.npz")


def test_oracle_is_the_reference_at_c2_scale():
    """The restated CPU twin reproduces reprojection() bitwise on the C2
    workload (25 cm, 512x512x200, half-fan, 90 bins; the committed fixture
    from the reference's own code) on two row bands of the sampled columns."""
    from measure.workloads import c2_workload, native_spectrum, native_tables
    from tests.shipped import volume_checksum
    gold = np.load(GOLD_C2)
    w = c2_workload()
    g = w["g"]
    assert int(gold["volume_checksum"]) == volume_checksum(w["vol"])
    mu, pdf = native_spectrum(w["spectrum_csv"])
    tabs = native_tables(w)
    views, cols = [int(v) for v in gold["views"]], gold["cols"]
    for rows in ((0, 12), (194, 206)):
        r = O.mbfpa_sampled(g, tabs, w["vol"], mu, pdf, w["xfactor"], views, cols, want=("f",),
                            ties=O.TIES_CPU, with_leng=False, flip=False, exact=True, rows=rows)["f"]
        assert np.array_equal(r[:, rows[0]:rows[1]], gold["out"][:, rows[0]:rows[1]])


def test_oracle_is_the_reference_on_the_shipped_decks(tmp_path):
    """The same on the reference's shipped decks (water-phantom slices with
    the repeat-last-slice rule, the shipped 101-bin spectrum), with the
    inputs built by the reference's own loader, spectrum and table code."""
    from tests import shipped
    if not (O.have_reference() and shipped.available()):
        pytest.skip("reference objects or staged data not built")
    gold = np.load(GOLD_DECKS)
    pdir, _ = shipped.layout(str(tmp_path))
    for tag, deck in (("d36", shipped.DECK_36), ("d360", shipped.DECK_360)):
        d = shipped.projector_inputs(pdir, deck)
        assert int(gold[f"{tag}_volume_checksum"]) == shipped.volume_checksum(d["vol"])
        views, cols = [int(v) for v in gold[f"{tag}_views"]], gold[f"{tag}_cols"]
        rows = (190, 210)
        r = O.mbfpa_sampled(d["g"], d["tabs"], d["vol"], d["mu"], d["pdf"], d["xfactor"], views, cols,
                            want=("f",), ties=O.TIES_CPU, with_leng=False, flip=False, exact=True,
                            rows=rows)["f"]
        assert np.array_equal(r[:, rows[0]:rows[1]], gold[f"{tag}_out"][:, rows[0]:rows[1]])
