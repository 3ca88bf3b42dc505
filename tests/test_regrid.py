"""Regridding pieces of the product, CPU side.

bsam_host_new_subgrids (the native library's Berger-Rigoutsos clustering,
host code) against the boxes the reference's own NewSubGrids makes
(tests/golden/ref_subgrids_*.npz, from its Fortran source): the same boxes
in the same order.  Also: every flagged cell covered, boxes disjoint, sides
at least minimumgridpoints, and nothing made from no flags.
"""
import os

import numpy as np
import pytest

from bsam_b200 import amr

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("n", [0, 1, 2, 3])
def test_new_subgrids_match_reference(gpu_free_lib, n):
    d = np.load(os.path.join(GOLD, f"ref_subgrids_{n}.npz"))
    nd = int(d["ndims"])
    got = amr.new_subgrids(d["flags"], float(d["fill"]), int(d["mgp"]))
    assert np.array_equal(got[:, :nd, :], d["boxes"][:, :nd, :])


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_new_subgrids_partition(gpu_free_lib, oracle, seed):
    rng = np.random.default_rng(seed)
    fl = (rng.random((48, 40)) < 0.04).astype(np.uint8)
    fl[10:20, 5:30] = 1
    boxes = amr.new_subgrids(fl, 0.85, 4)
    cov = np.zeros(fl.shape, dtype=int)
    for b in boxes:
        cov[b[0, 0] - 1:b[0, 1], b[1, 0] - 1:b[1, 1]] += 1
        assert min(b[0, 1] - b[0, 0], b[1, 1] - b[1, 0]) + 1 >= 4
    assert np.all(cov[fl == 1] == 1) and cov.max() == 1
    # the oracle's restatement agrees
    assert np.array_equal(oracle.new_subgrids(fl, 0.85, 4)[:, :2], boxes[:, :2])


def test_new_subgrids_nothing_flagged(gpu_free_lib):
    assert amr.new_subgrids(np.zeros((16, 16), dtype=np.uint8), 0.9, 4).shape[0] == 0
