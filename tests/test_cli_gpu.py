"""The command-line drivers (vcbct_proj, vcbct_cbct2: the reference's proj.exe
and cbct2 programs) end to end from txt decks, flexmaps, slice files and a
spectrum: the projections against the FP64 oracle, the filtered sinogram and
the short volume against the oracle's and the reference's FDK."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O
from virtualcbct_b200 import ProjGeometry, attenuation_table, decks, phantoms, trig_tables

pytestmark = pytest.mark.gpu

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
BIN = os.path.join(ROOT, "virtualcbct_b200", "bin")
DATA = os.path.join(ROOT, "virtualcbct_b200", "data")


def _run(prog, deck, cwd):
    exe = os.path.join(BIN, prog)
    if not os.path.exists(exe):
        pytest.fail(f"{exe} is not built (make -C virtualcbct_b200/csrc)")
    env = dict(os.environ, VCBCT_XRAYDB=os.path.join(DATA, "xraydb_mini"))
    r = subprocess.run([exe, deck], cwd=cwd, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    return r


def test_proj_then_cbct2_from_decks(cuda, tmp_path, monkeypatch):
    tmp = str(tmp_path)
    monkeypatch.chdir(tmp)  # deck paths are relative to the current directory
    N, slices, z_ic, V, W, H = 48, 40, 20, 36, 40, 32
    s, step = 0.2, 0.5
    vol_all = phantoms.ellipsoid_phantom(N, slices, s, step, seed=11)
    for i in range(slices):
        vol_all[i].tofile(os.path.join(tmp, f"elem_{i:03d}.raw"))
    shutil.copy(os.path.join(DATA, "spectrum_kramers100_90.csv"), os.path.join(tmp, "spec.csv"))
    angles = np.array([float(f"{a:.5f}") for a in phantoms.view_angles(V)])
    decks.write_flexmap(os.path.join(tmp, "views.flexmap"), angles)
    decks.write_proj_deck(os.path.join(tmp, "proj.txt"), spectrum="spec.csv", total_proj=V, proj_width=W,
                          proj_height=H, angle_file="views.flexmap", mat_prefix="elem", z_ic=z_ic,
                          output_name="proj_out", scale=(s, s, step), recon_size=N, recon_slices=slices,
                          mat_num=6, mat_type="human", xfactor=1000.0, reg=(0.0, 0.0, 0.0))
    _run("vcbct_proj", "proj.txt", tmp)
    got = np.fromfile(os.path.join(tmp, "proj_out.raw"), np.float32).reshape(V, H, W)

    d = decks.read_proj_deck(os.path.join(tmp, "proj.txt"))
    vol = vol_all[d["slice_first"]: d["slice_first"] + d["used_slices"]]
    g = ProjGeometry(N=N, Z=d["used_slices"], s=s, step=step, W=W, H=H, V=V, z_reg=d["z_reg"])
    ang = angles * 3.141592653589793238462643383279 / 180.0
    tabs = trig_tables(W, H, ang, np.zeros(V), np.zeros(V), g.pdet, g.dpn)
    mu, pdf = attenuation_table(os.path.join(tmp, "spec.csv"), os.path.join(DATA, "xraydb_mini"), 6)
    ref = O.mbfpa_forward(g, tabs, vol, mu, pdf, 1000.0, exact=True, want=("d",))["d"]
    rel = np.abs(got.astype(np.float64) - ref) / ref
    assert rel.max() <= 1e-5, f"max rel err {rel.max():.3e}"

    # FDK of those projections through the second program (increasing angles:
    # the deck reader reverses the view list, as the reference's loader does)
    decks.write_fdk_deck(os.path.join(tmp, "fdk.txt"), energy_class="kV", total_proj=V, proj_width=W,
                         proj_height=H, proj_header_bytes=0, proj_prefix="proj_out", proj_num_digits=8,
                         proj_first_number="hore", proj_ext="raw", angle_file="views.flexmap",
                         recon_size=27, target_class="*", recon_offset=-2, recon_step=0.25, recon_slices=12,
                         recon_scale=0.2, xfactor=1000, recon_file="fdk_vol.raw")
    _run("vcbct_cbct2", "fdk.txt", tmp)
    fd = decks.read_fdk_deck(os.path.join(tmp, "fdk.txt"))
    assert fd["reversed"] == 1
    filt = np.fromfile(os.path.join(tmp, "fltsngrm.raw"), np.float32).reshape(V, H, W)
    consts = O.fdk_consts(fd["det_pitch_iso_cm"])
    f64 = O.filter_sinogram(got, fd["xshift"], fd["yshift"], consts, mode=1)
    assert np.abs(filt - f64).max() <= 1e-5 * np.abs(f64).max()
    vi = np.fromfile(os.path.join(tmp, "fdk_vol.raw"), np.int16).reshape(fd["recon_slices"], 27, 27)
    if O.have_reference():
        rf, _ = O.ref_filter(got, fd["xshift"], fd["yshift"], fd["det_pitch_iso_cm"])
        rv, _ = O.ref_backproject(27, fd["recon_slices"], fd["recon_offset"], fd["recon_step"],
                                  fd["recon_scale"], rf, fd["xfactor"], fd["angles_rad"], fd["xshift"],
                                  fd["det_pitch_iso_cm"])
    else:
        rf = O.filter_sinogram(got, fd["xshift"], fd["yshift"], consts, mode=0)
        rv = O.backproject(27, fd["recon_slices"], fd["recon_offset"], fd["recon_step"], fd["recon_scale"],
                           rf, fd["xfactor"], fd["angles_rad"], fd["xshift"], consts)
    diff = np.abs(vi.astype(np.int32) - rv.astype(np.int16).astype(np.int32))
    assert diff.max() <= 1, f"{(diff > 1).sum()} voxels differ by more than 1 LSB"
    assert np.abs(vi).max() > 0


def test_load_deck_streams_the_same_volume(cuda, tmp_path, monkeypatch):
    """Projector.load_deck (slabs of slices streamed to the GPU) loads what
    the host reader assembles, including the missing / short file rule."""
    import torch
    tmp = str(tmp_path)
    monkeypatch.chdir(tmp)
    N, slices, V, W, H = 40, 30, 4, 32, 24
    vol_all = phantoms.random_volume(N, slices, seed=4, hi=900)
    for i in range(slices):
        if i == 13:
            continue                                   # missing: repeats slice 12
        raw = vol_all[i].tobytes()
        if i == 17:
            raw = raw[: len(raw) // 2]                 # short: tail from slice 16
        open(os.path.join(tmp, f"elem_{i:03d}.raw"), "wb").write(raw)
    angles = np.array([float(f"{a:.5f}") for a in phantoms.view_angles(V)])
    decks.write_flexmap(os.path.join(tmp, "v.flexmap"), angles)
    decks.write_proj_deck(os.path.join(tmp, "p.txt"), spectrum="s.csv", total_proj=V, proj_width=W,
                          proj_height=H, angle_file="v.flexmap", mat_prefix="elem", z_ic=15, output_name="o",
                          scale=(0.25, 0.25, 0.5), recon_size=N, recon_slices=slices, mat_num=6, mat_type="human",
                          xfactor=1000.0, reg=(0.0, 0.0, 0.0))
    d = decks.read_proj_deck("p.txt")
    host_vol, bad = decks.load_proj_volume(d)
    g = ProjGeometry(N=N, Z=d["used_slices"], s=0.25, step=0.5, W=W, H=H, V=V, z_reg=d["z_reg"])
    ang = angles * 3.141592653589793238462643383279 / 180.0
    tabs = trig_tables(W, H, ang, np.zeros(V), np.zeros(V), g.pdet, g.dpn)
    mu, pdf = attenuation_table(os.path.join(DATA, "spectrum_kramers100_90.csv"), os.path.join(DATA, "xraydb_mini"), 6)
    from virtualcbct_b200 import Projector
    a, b = Projector(g, *tabs), Projector(g, *tabs)
    for p in (a, b):
        p.set_spectrum(mu, pdf, 1000.0)
    a.load_volume(host_vol)
    assert b.load_deck(d) == bad == 2
    assert torch.equal(a.forward(), b.forward())
