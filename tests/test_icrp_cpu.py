"""The jittered media / organ tables of the phantom generator against the
reference's own converter program (oracle/_ref/icrp_convert, built from
ICRPphantoms_2mmslice/To_material_distribution_for512_random.cpp) on its own
CSV tables and a synthetic organ-number volume: the element volumes agree
exactly, so the table builder draws the reference's rand() sequence in the
reference's order."""
import os

import numpy as np
import pytest

import oracle as O
from oracle.refpath import reference_path
from virtualcbct_b200.icrp import PhantomTables

ICRP = reference_path("ICRPphantoms_2mmslice")
pytestmark = pytest.mark.skipif(not (O.have_icrp_convert() and os.path.isdir(ICRP)),
                                reason="reference converter or its tables not available")


def test_tables_reproduce_the_reference_converter(tmp_path):
    media, organs = os.path.join(ICRP, "AM_media.csv"), os.path.join(ICRP, "AM_organs.csv")
    numbers = np.loadtxt(organs, delimiter=",", usecols=0).astype(np.int64)
    rng = np.random.default_rng(5)
    ids = rng.choice(numbers, size=(100, 271, 543)).astype(np.uint8)
    ref = O.ref_icrp_convert(str(tmp_path), ids, media, organs)          # [6][Z][R][C]
    t = PhantomTables(media, organs, seed=1)                             # the reference's default seed
    ours = t.table[ids]                                                  # [Z][R][C][6]
    assert np.array_equal(ours.transpose(3, 0, 1, 2).view(np.int16), ref)
    # the jitter is real: a different seed gives different tables
    assert not np.array_equal(PhantomTables(media, organs, seed=2).table, t.table)
