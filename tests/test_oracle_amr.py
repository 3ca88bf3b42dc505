"""The oracle's AMR rows: Interpolate2D, GhostOverlap, SetGhost above the
root, and time stepping on a fixed hierarchy (CPU only).

Known answers from the reference's formulas: the coarse-fine ghost value is
the quadratic interpolant along a diagonal through two fine cells and one
coarse cell (a1 + a2 + a3 = 1 at offsets 2, 1, -1/2; boundary.f90:45-47), and
the end ghosts use a three-point fit along the face (b1 + b2 + b3 = 1), so
every ghost is exact for quadratic fields sampled at cell centres.
"""
import numpy as np
import pytest

from bsam_b200 import amr
from bsam_b200 import workloads as W


def quad(x, y):
    return 1.0 + 0.3 * x + 0.2 * y + 0.5 * x * x - 0.4 * x * y + 0.7 * y * y


def test_interpolate2d_exact_for_quadratics(oracle):
    hc = 1.0 / 16
    pmx = (16, 16)
    mb = (5, 12, 3, 10)  # fine patch over parent cells 5..12 x 3..10
    mx = (2 * (mb[1] - mb[0] + 1), 2 * (mb[3] - mb[2] + 1))
    hf = hc / 2
    I = np.arange(pmx[0] + 2)
    J = np.arange(pmx[1] + 2)
    XC, YC = np.meshgrid((I - 0.5) * hc, (J - 0.5) * hc, indexing="ij")
    qc = np.stack([quad(XC, YC), 2.0 * quad(XC, YC)], axis=-1)
    i = np.arange(mx[0] + 2)
    j = np.arange(mx[1] + 2)
    XF, YF = np.meshgrid((mb[0] - 1) * hc + (i - 0.5) * hf, (mb[2] - 1) * hc + (j - 0.5) * hf,
                         indexing="ij")
    exact = np.stack([quad(XF, YF), 2.0 * quad(XF, YF)], axis=-1)
    qf = exact.copy()
    qf[0, :, :] = qf[-1, :, :] = qf[:, 0, :] = qf[:, -1, :] = -7.0  # poison the ring
    for ipass in (1, 2):
        qf = oracle.interpolate2d(qf, qc, mb, (999, 999, 999, 999), ipass)
    ring = np.zeros(exact.shape[:2], bool)
    ring[0, :] = ring[-1, :] = ring[:, 0] = ring[:, -1] = True
    assert np.max(np.abs(qf[ring] - exact[ring])) < 1e-12
    assert np.array_equal(qf[~ring], exact[~ring])  # interior untouched


def test_interpolate2d_colours_and_physical_faces(oracle):
    rng = np.random.default_rng(3)
    qc = rng.random((18, 18, 2))
    qf = rng.random((10, 10, 2))
    red = oracle.interpolate2d(qf, qc, (3, 6, 3, 6), (999, 1, 999, 1), 1)
    black = oracle.interpolate2d(qf, qc, (3, 6, 3, 6), (999, 1, 999, 1), 2)
    both = oracle.interpolate2d(qf, qc, (3, 6, 3, 6), (999, 1, 999, 1), 0)
    changed_r = np.any(red != qf, axis=2)
    changed_b = np.any(black != qf, axis=2)
    assert not np.any(changed_r & changed_b)          # each ghost has one colour
    assert np.array_equal(np.where(changed_r[..., None], red, black), both)
    # Physical faces 2 and 4 (i = mx+1, j = my+1): only their corners move.
    assert not np.any((changed_r | changed_b)[-1, 1:-1])
    assert not np.any((changed_r | changed_b)[1:-1, -1])
    # Internal faces: every face ghost is set by one of the colours.
    assert np.all((changed_r | changed_b)[0, 1:-1]) and np.all((changed_r | changed_b)[1:-1, 0])


def test_hierarchy_without_refinement_equals_uniform(oracle):
    h = amr.build(32, [], eps=0.02, dt=1e-4, qerrortol=1e-9, field="wave")
    got = oracle.run_hier(h, 2)
    prob = W.Problem(ndims=2, mx=(32, 32, 1), eps=0.02, dt=1e-4, nsteps=2, qerrortol=1e-9,
                     c0=h.q0s[0][1:-1, 1:-1, 0].ravel(order="F"))
    ref = oracle.run_uniform(prob, nsteps=2, q0=h.q0s[0])
    assert np.array_equal(got["q"][0], ref["q"][-1])
    assert np.array_equal(got["nvcycles"], ref["nvcycles"])


@pytest.mark.parametrize("boxes", [
    [(1, (9, 9), (16, 16))],
    [(1, (9, 9), (16, 16)), (1, (25, 9), (16, 16)), (2, (21, 21), (16, 16))],
])
def test_amr_hierarchy_converges(oracle, boxes):
    h = amr.build(32, boxes, eps=0.04, dt=5e-5, qerrortol=1e-9)
    got = oracle.run_hier(h, 2)
    assert np.all(got["residual"] < h.qerrortol), got
    assert np.all(np.isfinite(np.concatenate([q.ravel() for q in got["q"]])))
    # Siblings agree across their shared face: the ghost of one equals the
    # neighbour's interior cell (GhostOverlap).
    if len(boxes) > 1:
        qa, qb = got["q"][1], got["q"][2]  # patches at global x 9..24 and 25..40
        assert np.array_equal(qa[-1, 1:-1, :], qb[1, 1:-1, :])
        assert np.array_equal(qb[0, 1:-1, :], qa[-2, 1:-1, :])
