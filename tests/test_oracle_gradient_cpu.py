"""Pins the FP64 gradient oracle (the adjoint has no reference counterpart):
orc_mbfpa_adjoint against central differences of the FP64 forward oracle,
on the CPU.  The GPU adjoint is then checked against this oracle
(tests/test_adjoint_gpu.py, tests/test_materials_gpu.py)."""
import numpy as np
import pytest

import oracle as O
from tests.cases import spectrum
from virtualcbct_b200 import ProjGeometry, phantoms, trig_tables


def _case(nmat, seed, z_reg):
    g = ProjGeometry(N=24, Z=8, s=0.4, step=0.6, W=20, H=16, V=3, dpn=480.0, z_reg=z_reg, nmat=nmat)
    ang = np.deg2rad(phantoms.view_angles(g.V))
    tabs = trig_tables(g.W, g.H, ang, np.zeros(g.V), np.zeros(g.V), g.pdet, g.dpn)
    rng = np.random.default_rng(seed)
    volf = rng.uniform(50.0, 900.0, size=(g.Z, nmat, g.N, g.N)).astype(np.float32)
    mu6, pdf = spectrum()
    mu = np.stack([mu6[k % 6] * np.float32(1.0 + 0.15 * (k // 6)) for k in range(nmat)]).astype(np.float32)
    resid = rng.normal(size=(g.V, g.H, g.W))
    return g, tabs, volf, mu, pdf, resid


@pytest.mark.parametrize("nmat,seed,z_reg", [(6, 0, 0.3), (6, 1, 0.0), (2, 2, 0.3), (8, 3, 0.3)])
def test_gradient_oracle_matches_central_differences(nmat, seed, z_reg):
    g, tabs, volf, mu, pdf, resid = _case(nmat, seed, z_reg)
    grad = O.mbfpa_adjoint(g, tabs, volf, mu, pdf, 1000.0, resid)

    def loss(v):
        d = O.mbfpa_forward(g, tabs, None, mu, pdf, 1000.0, volf=v, exact=False, want=("d",))["d"]
        return float(np.sum(resid * d))

    rng = np.random.default_rng(100 + seed)
    cand = np.argwhere(np.abs(grad) > 1e-3 * np.abs(grad).max())
    pick = cand[rng.choice(len(cand), size=24, replace=False)]
    h = 2.0 ** -6  # v +- h is exact in float32 for |v| < 2^17
    errs = []
    for idx in map(tuple, pick):
        vp = volf.copy()
        vm = volf.copy()
        vp[idx] += np.float32(h)
        vm[idx] -= np.float32(h)
        fd = (loss(vp) - loss(vm)) / (2 * h)
        errs.append(abs(fd - grad[idx]) / abs(grad[idx]))
    # voxels no ray crosses have no gradient
    assert np.abs(grad).max() > 0 and len(cand) >= 24
    assert np.median(errs) <= 1e-5 and np.max(errs) <= 1e-3, (np.median(errs), np.max(errs))
