"""The seeded synthetic inputs that stand in for the reference's phantoms:
encoding (fraction x density x 1000 per element), tissue densities and
jitter of the ellipsoid phantom, the water cylinder, view lists and spectra."""
import numpy as np

from virtualcbct_b200 import phantoms as P


def test_water_cylinder_encoding():
    N, s, r = 40, 0.5, 7.0
    vol = P.water_cylinder(N, 3, s, r)
    assert vol.shape == (3, 6, N, N) and vol.dtype == np.uint16
    c = (np.arange(N) - (N - 1) / 2.0) * s
    inside = c[None, :] ** 2 + c[:, None] ** 2 <= r * r
    for z in range(3):
        assert np.all(vol[z, 0][inside] == 111) and np.all(vol[z, 3][inside] == 889)
        assert np.all(vol[z, 2][~inside] == 1)  # air: N at 0.0012 g/cm3 x 1000
        assert np.all(vol[z, 2][inside] == 0)
        for k in (1, 4, 5):
            assert not vol[z, k].any()
        assert not vol[z, 0][~inside].any()


def test_ellipsoid_phantom_classes_densities_and_jitter():
    N, Z, s, step = 72, 6, 0.5, 1.0
    v = P.ellipsoid_phantom(N, Z, s, step, seed=3, as_float=True).astype(np.float64)
    assert v.shape == (Z, 6, N, N)
    rho = v.sum(axis=1) / 1000.0           # fractions close to 1: the voxel's density
    air = (v[:, 2] == np.float32(1.2)) & (v.sum(axis=1) == np.float32(1.2))
    tissue = ~air
    got = np.unique(np.round(rho[tissue], 4))
    assert set(got) <= {1.0, 0.95, 0.26, 1.92}
    assert {1.0, 0.26, 1.92} <= set(got)
    # per-element jitter within +-5 % of the class's base fraction (O closes the sum)
    for name, d in (("soft", 1.0), ("lung", 0.26), ("bone", 1.92), ("fat", 0.95)):
        m = tissue & (np.abs(rho - d) < 1e-4)
        if not m.any():
            continue
        base = np.asarray(P.TISSUE[name])
        for k in (0, 1, 2, 4, 5):
            if base[k] == 0:
                assert not v[:, k][m].any()
                continue
            f = v[:, k][m] / (d * 1000.0)
            assert f.min() >= base[k] * 0.95 - 1e-6 and f.max() <= base[k] * 1.05 + 1e-6
    # body 30 x 22 cm: tissue spans about +-15 cm in x and +-11 cm in y at the centre
    x = (np.arange(N) - (N - 1) / 2.0) * s
    cz = Z // 2
    cols = np.nonzero(tissue[cz].any(axis=0))[0]
    rows = np.nonzero(tissue[cz].any(axis=1))[0]
    assert abs(x[cols].max() - 15.0) <= 1.0 and abs(x[rows].max() - 11.0) <= 1.0


def test_ellipsoid_phantom_is_seeded():
    a = P.ellipsoid_phantom(48, 4, 0.7, 1.0, seed=5)
    b = P.ellipsoid_phantom(48, 4, 0.7, 1.0, seed=5)
    c = P.ellipsoid_phantom(48, 4, 0.7, 1.0, seed=6)
    assert a.dtype == np.uint16 and np.array_equal(a, b) and not np.array_equal(a, c)


def test_view_angles_and_spectrum():
    a = P.view_angles(36)
    assert a[0] == -170.0001 and np.allclose(np.diff(a), 10.0)
    lo, hi, f = P.kramers_spectrum(100.0)
    assert np.allclose(hi - lo, 0.001) and lo[0] == 0.010 and np.isclose(f.sum(), 1.0)
    assert np.all(f >= 0) and f[-1] < f[0]
    text = P.spectrum_csv_text(lo, hi, f)
    assert text.splitlines()[0] == "Energy,1000,Fraction" and len(text.splitlines()) == len(f) + 1
