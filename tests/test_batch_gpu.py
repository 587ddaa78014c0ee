"""Batched projection: uneven phantoms in one persistent launch, in one flat
launch or as per-item launches on graph branches (and their CUDA-graph
replay) give exactly the per-phantom results, and each strategy's output of
every item agrees with the FP64 oracle; more items than one launch's
parameter block holds take several launches."""
import numpy as np
import pytest

import oracle as O
from tests.cases import proj_case, spectrum
from virtualcbct_b200 import Batch, Projector

pytestmark = pytest.mark.gpu


RTOL = 1e-5  # projections: relative, per detector pixel


def _projector(cuda, kind, seed, keep=False, **kw):
    import torch
    g, tabs, vol, _ = proj_case(kind, seed=seed, **kw)
    mu, pdf = spectrum()
    p = Projector(g, *tabs)
    p.set_spectrum(mu, pdf, 1000.0)
    p.load_volume(torch.from_numpy(vol.view(np.int16)).to(cuda))
    if keep:
        p.case = (g, tabs, vol, mu, pdf)
    return p


def test_every_strategy_matches_the_fp64_oracle(cuda):
    import torch
    ps = [_projector(cuda, "ellipsoid", 5, keep=True, N=48, Z=12, V=3, W=40, H=36),
          _projector(cuda, "random", 6, keep=True, N=40, Z=20, V=2, W=33, H=41, xshift=0.4),
          _projector(cuda, "water", 0, keep=True, N=56, Z=10, V=4, W=24, H=24)]
    refs = []
    for p in ps:
        g, tabs, vol, mu, pdf = p.case
        refs.append(O.mbfpa_forward(g, tabs, vol, mu, pdf, 1000.0, exact=False, want=("d",))["d"])
    b = Batch()
    outs = [b.add(p) for p in ps]
    for strategy in (Batch.PERSISTENT, 1, Batch.FLAT):
        b.configure(strategy, 4)
        for o in outs:
            o.fill_(float("nan"))
        b.forward(use_graph=True)
        torch.cuda.synchronize()
        for o, ref in zip(outs, refs):
            got = o.cpu().numpy().astype(np.float64)
            assert np.isfinite(got).all()
            assert np.max(np.abs(got - ref) / ref) <= RTOL, strategy


def test_more_items_than_one_launch_holds(cuda):
    """45 items: the single-launch strategies split them into launches of at
    most 40 (the parameter block's capacity)."""
    import torch
    ps = [_projector(cuda, "random", 100 + i, N=16, Z=4 + i % 5, V=1 + i % 3, W=8 + i % 4, H=6) for i in range(45)]
    plain = [p.forward().cpu().numpy() for p in ps]
    b = Batch()
    outs = [b.add(p) for p in ps]
    for strategy in (Batch.PERSISTENT, Batch.FLAT):
        b.configure(strategy, 2)
        for o in outs:
            o.fill_(float("nan"))
        b.forward(use_graph=True)
        torch.cuda.synchronize()
        for o, ref in zip(outs, plain):
            assert np.array_equal(o.cpu().numpy(), ref), strategy


def test_batched_equals_plain_launches(cuda):
    import torch
    ps = [_projector(cuda, "ellipsoid", 1, N=64, Z=20, V=5),
          _projector(cuda, "random", 2, N=48, Z=9, V=2, W=36, H=70),
          _projector(cuda, "water", 0, N=80, Z=33, V=7, W=52, H=44),
          _projector(cuda, "random", 3, N=32, Z=64, s=0.3, step=0.02, V=2, W=24, H=40, dpn=900.0)]
    plain = [p.forward().cpu().numpy() for p in ps]
    b = Batch()
    outs = [b.add(p) for p in ps]
    for strategy, cpb in ((0, 4), (1, 4), (2, 4), (0, 2), (1, 8), (2, 8), (2, 2)):
        b.configure(strategy, cpb)
        for use_graph in (False, True, True):
            for o in outs:
                o.fill_(float("nan"))
            b.forward(use_graph=use_graph)
            torch.cuda.synchronize()
            for o, ref in zip(outs, plain):
                assert np.array_equal(o.cpu().numpy(), ref), (strategy, cpb, use_graph)
    c = b.autotune()
    assert c % 100 in (2, 4, 8) and c // 100 in (0, 1, 2)
    b.forward(use_graph=True)
    torch.cuda.synchronize()
    for o, ref in zip(outs, plain):
        got = o.cpu().numpy()
        assert np.max(np.abs(got - ref) / ref) <= 1e-6


def test_projector_autotune_keeps_results(cuda):
    p = _projector(cuda, "ellipsoid", 4)
    ref = p.forward().cpu().numpy()
    c = p.autotune()
    assert c in (2, 4, 8)
    assert np.max(np.abs(p.forward().cpu().numpy() - ref) / ref) <= 1e-6
