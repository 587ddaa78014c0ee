"""Iterative-reconstruction helpers: the oracle restatements of lengthproj
and IR_ImageCBCT against the reference's own code (oracle/_ref), bitwise."""
import numpy as np
import pytest

import oracle as O
from tests.cases import proj_case

needs_ref = pytest.mark.skipif(not O.have_reference(), reason="oracle/_ref not built")


def ir_case(seed=0, N=24, Z=10, V=5, W=40, H=32, z_reg=0.3, xshift=0.0):
    g, tabs, _, _ = proj_case("random", N=N, Z=Z, V=V, W=W, H=H, z_reg=z_reg, seed=seed, xshift=xshift)
    rng = np.random.default_rng(seed)
    proj = rng.integers(20000, 65000, size=(V, H, W)).astype(np.uint16)
    return g, tabs, proj


@needs_ref
@pytest.mark.parametrize("ite,xshift,views", [(0, 0.0, None), (1, 1.2, (1, 4)), (0, -0.7, (0, 5))])
def test_lengthproj_oracle_is_the_reference(ite, xshift, views):
    g, tabs, proj = ir_case(seed=ite + 3, xshift=xshift)
    a = O.lengthproj(g, tabs, proj, ite=ite, views=views)
    b = O.ref_lengthproj(g, tabs, proj, ite=ite, views=views)
    assert np.array_equal(a, b)
    assert np.abs(a).max() > 0


@needs_ref
@pytest.mark.parametrize("wtv", [0.0, 0.002])
def test_ir_update_oracle_is_the_reference(wtv):
    rng = np.random.default_rng(11)
    N, Z = 20, 7
    before = rng.integers(0, 3000, size=(Z, N, N)).astype(np.int16)
    npf = rng.uniform(1.0, 5.0, size=(Z, N, N)).astype(np.float32)
    npf_re = rng.uniform(1.0, 5.0, size=(Z, N, N)).astype(np.float32)
    a = O.ir_update(N, Z, 0.1, before, npf, npf_re, 0.3, wtv, 0.0)
    b = O.ref_ir_update(N, Z, 0.1, before, npf, npf_re, 0.3, wtv, 0.0)
    assert np.array_equal(a, b)
