"""Phantom generator on the GPU: the organ-number -> element lookup kernel
against the table applied on the host, for host and device buffers, on
seeded synthetic media / organ tables in the reference's CSV formats."""
import numpy as np
import pytest

from virtualcbct_b200.icrp import PhantomTables, organs_to_elements

pytestmark = pytest.mark.gpu


def _tables(tmp_path, seed=3):
    rng = np.random.default_rng(seed)
    media = tmp_path / "media.csv"
    rows = []
    for i in range(1, 53):  # media are indexed by id - 1: ids 1..53
        w = rng.uniform(0, 20, size=13)
        w[4:6] = 0.0
        rows.append(",".join([str(i)] + [f"{x:.3f}" for x in w]))
    rows.append("53,0,0,70,30,0,0,0,0,0,0,0,0,0")  # air, not jittered
    media.write_text("\n".join(rows) + "\n")
    organs = tmp_path / "organs.csv"
    orows = [f"{k},{int(rng.integers(1, 53))},{rng.uniform(0.2, 1.9):.3f}" for k in range(1, 141)]
    orows.append("141,53,0.001")
    organs.write_text("\n".join(orows) + "\n")
    return PhantomTables(str(media), str(organs), seed=7)


def test_organs_to_elements_matches_host_lookup(cuda, tmp_path):
    import torch
    t = _tables(tmp_path)
    tab = t.table
    assert tab[141].tolist() == [0, 0, int(np.float32(70) * np.float32(0.001) * 10), int(np.float32(30) * np.float32(0.001) * 10), 0, 0]
    rng = np.random.default_rng(0)
    ids = rng.integers(0, 142, size=(7, 33, 45)).astype(np.uint8)   # 0: no organ row -> 0
    ref = tab[ids].transpose(0, 3, 1, 2)                             # [Z][6][R][C]
    host = organs_to_elements(ids, t)
    assert np.array_equal(host, ref)
    dev = organs_to_elements(torch.from_numpy(ids).to(cuda), t).cpu().numpy().view(np.uint16)
    assert np.array_equal(dev, ref)
    # slices of a multiple of 8 voxels take the 8-voxels-per-thread path
    ids8 = rng.integers(0, 256, size=(5, 32, 48)).astype(np.uint8)
    ref8 = tab[ids8].transpose(0, 3, 1, 2)
    dev8 = organs_to_elements(torch.from_numpy(ids8).to(cuda), t).cpu().numpy().view(np.uint16)
    assert np.array_equal(dev8, ref8)
    assert np.array_equal(organs_to_elements(ids8, t), ref8)
