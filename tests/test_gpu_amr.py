"""Refined (AMR) levels on the GPU against the oracle, 2D and 3D FP64 form.

Bar: after the time steps, phi and mu of every patch on every level >= 0
(ghost rings included) within 1e-11 of the oracle (relative, max norm),
identical V-cycle counts, residuals within 1e-9 relative.  The hierarchies
exercise coarse-fine interpolation on every face and colour (Interpolate2D,
Interpolate3D), sibling exchange across shared faces and corners
(GhostOverlap), patches that mix physical and internal faces, two refined
levels, and FillDown.  In 3D: user-coded faces, and physical faces coded 99,
which the edge check of Interpolate3D treats like internal ones
(boundary.f90:1354).
"""
import numpy as np
import pytest

from bsam_b200 import amr

pytestmark = pytest.mark.gpu

HIERS = {
    "one_patch": [(1, (9, 9), (16, 16))],
    "siblings_and_level2": [(1, (9, 9), (16, 16)), (1, (25, 9), (16, 16)),
                            (2, (21, 21), (16, 16))],
    "physical_faces": [(1, (1, 1), (16, 24)), (1, (17, 33), (32, 16)), (2, (1, 5), (12, 12))],
    "corner_neighbours": [(1, (9, 9), (12, 12)), (1, (21, 21), (12, 12)),
                          (1, (33, 9), (8, 8))],
}


@pytest.mark.parametrize("name", sorted(HIERS))
def test_amr_matches_oracle(gpu_lib, oracle, name):
    h = amr.build(32, HIERS[name], eps=0.04, dt=5e-5, qerrortol=1e-9)
    ref = oracle.run_hier(h, 2)
    with amr.HierSolver(h) as s:
        got = s.run(2)
    assert np.array_equal(got["nvcycles"], ref["nvcycles"]), (got["nvcycles"], ref["nvcycles"])
    assert np.allclose(got["residual"], ref["residual"], rtol=1e-9, atol=0), (
        got["residual"], ref["residual"])
    for k, (a, b) in enumerate(zip(got["q"], ref["q"])):
        for v in range(2):
            err = float(np.max(np.abs(a[..., v] - b[..., v])) / np.max(np.abs(b[..., v])))
            assert err < 1e-11, (name, k, v, err)


HIERS3 = {
    # (n_root, boxes, root face code)
    "one_patch_3d": (16, [(1, (9, 9, 9), (12, 12, 12))], 1),
    "siblings_level2_3d": (16, [(1, (5, 5, 5), (12, 12, 12)), (1, (17, 5, 5), (8, 12, 12)),
                                (2, (13, 13, 13), (8, 8, 8))], 1),
    "user_faces_3d": (16, [(1, (1, 1, 1), (10, 12, 8)), (1, (11, 1, 1), (6, 12, 8))], 10),
    "code99_3d": (16, [(1, (5, 1, 1), (12, 12, 10)), (1, (5, 13, 1), (12, 8, 10))], 99),
}


@pytest.mark.parametrize("name", sorted(HIERS3))
def test_amr3d_matches_oracle(gpu_lib, oracle, name):
    n, boxes, code = HIERS3[name]
    h = amr.build(n, boxes, eps=0.08, dt=5e-5, qerrortol=1e-9, mthbc=code, ndims=3,
                  field="wave", seed=5)
    ref = oracle.run_hier(h, 2)
    with amr.HierSolver(h) as s:
        got = s.run(2)
    assert np.array_equal(got["nvcycles"], ref["nvcycles"]), (got["nvcycles"], ref["nvcycles"])
    assert np.allclose(got["residual"], ref["residual"], rtol=1e-9, atol=0), (
        got["residual"], ref["residual"])
    for k, (a, b) in enumerate(zip(got["q"], ref["q"])):
        for v in range(2):
            err = float(np.max(np.abs(a[..., v] - b[..., v])) / np.max(np.abs(b[..., v])))
            assert err < 1e-11, (name, k, v, err)


def test_amr_bottom_kernel_off_is_identical(gpu_lib):
    h = amr.build(32, HIERS["siblings_and_level2"], eps=0.04, dt=5e-5, qerrortol=1e-9)
    with amr.HierSolver(h) as s:
        a = s.run(2)
    with amr.HierSolver(h, bottom_cells=-1) as s:
        b = s.run(2)
    for x, y in zip(a["q"], b["q"]):
        assert np.array_equal(x, y)
