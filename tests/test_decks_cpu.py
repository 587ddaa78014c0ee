"""Input decks (txt info files, flexmaps, slice files) read by the C library,
checked field by field against the reference's own loaders (oracle/_ref,
projectionData.cpp and projectionDataMVkV.cpp compiled from the reference)
when they are built, and against the loaders' rules written out here."""
import os

import numpy as np
import pytest

import oracle as O
from virtualcbct_b200 import _native as N
from virtualcbct_b200 import decks

PI = 3.141592653589793238462643383279
needs_ref = pytest.mark.skipif(not O.have_reference(), reason="oracle/_ref not built")


def _proj_deck(tmp, N_=16, slices=40, z_ic=20, mat=6, V=36, missing=(), short=(), start=-170.0001,
               zscale=0.2):
    rng = np.random.default_rng(3)
    for i in range(slices):
        if i in missing:
            continue
        a = rng.integers(0, 2000, size=(mat, N_, N_)).astype(np.uint16)
        raw = a.tobytes()
        if i in short:
            raw = raw[: len(raw) // 3]
        with open(os.path.join(tmp, f"elem_{i:03d}.raw"), "wb") as f:
            f.write(raw)
    decks.write_flexmap(os.path.join(tmp, "views.flexmap"), start + 10.0 * np.arange(V),
                        xshift=0.3, yshift=-0.1)
    decks.write_proj_deck(os.path.join(tmp, "proj.txt"), spectrum="spec.csv", total_proj=V,
                          proj_width=40, proj_height=32, angle_file="views.flexmap", mat_prefix="elem",
                          z_ic=z_ic, output_name="out_proj", scale=(0.1, 0.1, zscale), recon_size=N_,
                          recon_slices=slices, mat_num=mat, mat_type="human", xfactor=1000.0,
                          reg=(0.25, -0.5, 0.75))
    return os.path.join(tmp, "proj.txt")


def _window(N_, y_scale, z_scale, z_ic, slices):
    # projectionData.cpp:173-185 with physParams.h:47-51
    z_length = (100.0 + (N_ // 2) * y_scale) / (53.8 + 100.0) * 0.05 * 800.0
    iz = int(z_length / z_scale)
    lo = max(0, z_ic - (iz // 2 + 1))
    hi = min(z_ic + (iz // 2 + 1), slices)
    return lo, hi


def test_proj_deck_fields_and_slice_window(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    txt = _proj_deck(str(tmp_path), slices=30, z_ic=12)
    d = decks.read_proj_deck(txt)
    assert d["spectrum"] == "spec.csv" and d["output_name"] == "out_proj" and d["mat_type"] == "human"
    assert (d["total_proj"], d["proj_width"], d["proj_height"], d["recon_size"]) == (36, 40, 32, 16)
    assert (d["x_reg"], d["y_reg"], d["z_reg_file"]) == (0.25, -0.5, 0.75)
    lo, hi = _window(16, 0.1, 0.2, 12, 30)
    assert (d["slice_first"], d["used_slices"], d["z_ic_local"]) == (lo, hi - lo, 12 - lo)
    assert d["z_reg"] == ((hi - lo) // 2 - (12 - lo)) * 0.2
    vol, bad = decks.load_proj_volume(d)
    assert bad == 0 and vol.shape == (hi - lo, 6, 16, 16)
    raw = np.fromfile(f"elem_{lo:03d}.raw", np.uint16).reshape(6, 16, 16)
    assert np.array_equal(vol[0], raw)
    a, x, y = decks.read_flexmap("views.flexmap", 36)
    written = np.array([float(f"{v:.5f}") for v in -170.0001 + 10.0 * np.arange(36)])
    assert np.array_equal(a, written * PI / 180.0)
    assert np.all(x == 0.3) and np.all(y == -0.1)


@needs_ref
@pytest.mark.parametrize("z_ic,zscale", [(20, 0.2), (2, 0.2), (38, 0.5), (20, 0.05)])
def test_proj_deck_matches_reference_loader(tmp_path, monkeypatch, z_ic, zscale):
    monkeypatch.chdir(tmp_path)
    txt = _proj_deck(str(tmp_path), z_ic=z_ic, zscale=zscale, missing=(z_ic,), short=(z_ic + 1,))
    ref = O.ref_proj_load(txt)
    d = decks.read_proj_deck(txt)
    for k in ("total_proj", "proj_width", "proj_height", "recon_size", "recon_slices", "mat_num",
              "used_slices", "z_ic_local", "x_scale", "y_scale", "z_scale", "xfactor", "x_reg", "y_reg",
              "det_pitch_cm", "det_pitch_iso_cm", "sad_cm", "det_pixel_num", "det_iso_cm", "spectrum",
              "output_name", "mat_type"):
        assert d[k] == ref[k], k
    vol, bad = decks.load_proj_volume(d)
    # a missing slice repeats the previous one; a short file overwrites its head
    assert bad == 2
    assert np.array_equal(vol, ref["volume"])
    a, x, y = decks.read_flexmap(d["angle_file"], d["total_proj"])
    assert np.array_equal(a, ref["angles_rad"]) and np.array_equal(x, ref["xshift"])
    assert np.array_equal(y, ref["yshift"])


def _fdk_deck(tmp, angles, classes="0", target="*", energy="kV", first="hore", offset=-5, step=0.1,
              slices=100, V=None, H=400):
    V = len(angles) if V is None else V
    decks.write_flexmap(os.path.join(tmp, "fdk.flexmap"), angles, xshift=np.linspace(0, 20, len(angles)),
                        yshift=0.5, classes=classes)
    decks.write_fdk_deck(os.path.join(tmp, "fdk.txt"), energy_class=energy, total_proj=V, proj_width=40,
                         proj_height=H, proj_header_bytes=0, proj_prefix="proj_in", proj_num_digits=8,
                         proj_first_number=first, proj_ext="raw", angle_file="fdk.flexmap", recon_size=27,
                         target_class=target, recon_offset=offset, recon_step=step, recon_slices=slices,
                         recon_scale=0.1, xfactor=1000, recon_file="fdk_out.raw")
    return os.path.join(tmp, "fdk.txt")


def test_fdk_deck_rules(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    up = np.array([float(f"{v:.5f}") for v in -180.0001 + 10.0 * np.arange(36)])
    d = decks.read_fdk_deck(_fdk_deck(str(tmp_path), up))
    # increasing angles: 1st - 30th < 0 -> reversed (projectionDataMVkV.cpp:184-197)
    assert d["reversed"] == 1 and d["n_target"] == 36 and d["n_lines"] == 36
    assert np.array_equal(d["angles_rad"], up[::-1] * PI / 180.0)
    assert d["proj_first_number"] == 0 and d["det_pitch_iso_cm"] == 0.032509752
    assert d["recon_slices"] == 100 and d["proj_prefix"] == "proj_in" and d["proj_ext"] == "raw"
    d = decks.read_fdk_deck(_fdk_deck(str(tmp_path), up[::-1], first="1A"))
    assert d["reversed"] == 0 and d["proj_first_number"] == 0x1A
    assert np.array_equal(d["angles_rad"], up[::-1] * PI / 180.0)
    # class filter: only class "1" views, in (reversed) order; the rest stay zero
    cls = ["1" if i % 3 == 0 else "2" for i in range(36)]
    d = decks.read_fdk_deck(_fdk_deck(str(tmp_path), up, classes=cls, target="1"))
    keep = [a for a, c in zip(up[::-1], cls[::-1]) if c == "1"]
    assert d["n_target"] == 12 and np.array_equal(d["angles_rad"][:12], np.array(keep) * PI / 180.0)
    assert np.all(d["angles_rad"][12:] == 0.0)
    # slice-count correction: offset + step * (slices - 1) >= proj_height (cm vs pixels)
    d = decks.read_fdk_deck(_fdk_deck(str(tmp_path), up, offset=10, step=0.5, slices=100, H=40))
    assert d["recon_slices"] == int((40 - 10) / 0.5)
    d = decks.read_fdk_deck(_fdk_deck(str(tmp_path), up, offset=5, step=-0.5, slices=100))
    assert d["recon_slices"] == int((5 + 1) / 0.5)
    # panel offset class from the mean xshift (0..20 -> mean 10 -> M)
    assert d["panel_class"] == "M"


def test_fdk_deck_errors(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    up = -180.0001 + 10.0 * np.arange(36)
    with pytest.raises(N.VcbctError) as e:
        decks.read_fdk_deck(_fdk_deck(str(tmp_path), up, energy="keV"))
    assert e.value.code == 1
    with pytest.raises(N.VcbctError) as e:
        decks.read_fdk_deck(_fdk_deck(str(tmp_path), up, V=20))  # 36 matching > 20 views
    assert e.value.code == 3
    with pytest.raises(N.VcbctError) as e:
        decks.read_flexmap("fdk.flexmap", 10)
    assert e.value.code == 3
    with open("bad.flexmap", "w") as f:
        f.write("10.0 0 0 0\n20.0 zero 0 0\n")
    with pytest.raises(N.VcbctError) as e:
        decks.read_flexmap("bad.flexmap", 10)
    assert e.value.code == 5
    with pytest.raises(N.VcbctError) as e:
        decks.read_proj_deck("no_such_deck.txt")
    assert e.value.code == 5


@needs_ref
@pytest.mark.parametrize("case", ["up", "down", "filtered", "fewer_lines", "slices"])
def test_fdk_deck_matches_reference_loader(tmp_path, monkeypatch, case):
    monkeypatch.chdir(tmp_path)
    up = -180.0001 + 10.0 * np.arange(36)
    kw = {}
    if case == "down":
        angles = up[::-1]
    elif case == "filtered":
        angles, kw = up, dict(classes=["1" if i % 2 else "2" for i in range(36)], target="2")
    elif case == "fewer_lines":
        angles, kw = up, dict(V=40)
    elif case == "slices":
        angles, kw = up, dict(offset=10, step=0.5, slices=100, H=40)
    else:
        angles = up
    txt = _fdk_deck(str(tmp_path), angles, **kw)
    ref = O.ref_fdk_load(txt)
    d = decks.read_fdk_deck(txt)
    assert d["n_target"] == ref["n_target"] == ref["ret"]
    for k in ("total_proj", "proj_width", "proj_height", "recon_size", "recon_offset", "recon_slices",
              "xfactor", "recon_step", "recon_scale", "det_pitch_iso_cm", "proj_prefix", "proj_ext",
              "recon_file", "panel_class"):
        assert d[k] == ref[k], k
    for k in ("angles_rad", "xshift", "yshift"):
        assert np.array_equal(d[k], ref[k]), k
