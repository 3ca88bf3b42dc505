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


def _level(nd, rng):
    """Three disjoint patches of one level (two of them side by side) in a
    48^d index space, with random flags: descs and flags."""
    if nd == 2:
        boxes = [((1, 1), (16, 12)), ((17, 1), (10, 12)), ((5, 25), (20, 14))]
    else:
        boxes = [((1, 1, 1), (10, 8, 6)), ((11, 1, 1), (6, 8, 6)), ((3, 13, 9), (8, 6, 10))]
    descs, flags = [], []
    for lo, sz in boxes:
        mg = [[lo[k], lo[k] + sz[k] - 1] for k in range(nd)] + [[1, 1]] * (3 - nd)
        descs.append({"level": 1, "parent": 0, "mx": list(sz) + [1] * (3 - nd),
                      "mbounds": [[1, 1]] * 3, "mglobal": mg, "mthbc": [999] * 6,
                      "dx": 1.0, "xlower": [0.0] * 3})
        flags.append((rng.random(sz) < 0.03).astype(np.uint8))
    return descs, flags


@pytest.mark.parametrize("nd,ibuffer", [(2, 1), (2, 2), (3, 1)])
def test_buffer_flags_match_oracle(gpu_free_lib, oracle, nd, ibuffer):
    """bsam_host_buffer_flags against the oracle's restatement of
    BufferAndList + InflateEdgeTags (buffers cross into neighbour patches)."""
    rng = np.random.default_rng(7 + nd + ibuffer)
    descs, flags = _level(nd, rng)
    flags[0][(-1,) + (0,) * (nd - 1)] = 1   # at the shared face of patches 0 and 1
    got = amr.buffer_flags(nd, descs, flags, ibuffer)
    want = oracle.buffer_flags(nd, descs, flags, ibuffer)
    for g, w, f in zip(got, want, flags):
        assert np.array_equal(g, w)
        assert np.all(g[f == 1] == 1)
    assert got[1][(0,) * nd] == 1           # the neighbour got the buffer
    assert all(np.array_equal(g, f) for g, f in zip(amr.buffer_flags(nd, descs, flags, 0), flags))


@pytest.mark.parametrize("nd", [2, 3])
def test_child_desc_matches_oracle(gpu_free_lib, oracle, nd):
    """bsam_host_child_desc (MakeNewGrid's geometry) against the oracle's
    restatement, for boxes inside, and touching each face of, a parent."""
    rng = np.random.default_rng(nd)
    mx = [12, 10, 8][:nd]
    parent = {"level": 1, "parent": 0, "mx": mx + [1] * (3 - nd), "mbounds": [[1, 1]] * 3,
              "mglobal": [[5, 4 + mx[k]] for k in range(nd)] + [[1, 1]] * (3 - nd),
              "mthbc": [1, 999, 999, 1, 1, 999][:2 * nd] + [1] * (6 - 2 * nd),
              "dx": 0.125, "xlower": [0.5, 0.375, 0.25][:nd] + [0.0] * (3 - nd)}
    for _ in range(20):
        box = []
        for k in range(nd):
            a, b = sorted(rng.integers(1, mx[k] + 1, size=2))
            box += [int(a), int(b)]
        got = amr.child_desc(nd, parent, 3, box)
        want = oracle.child_desc(nd, parent, 3, box)
        assert got == want, (box, got, want)


def test_regrid_run_on_oracle(oracle):
    """The regrid driver (amr.RegridRun) over the oracle backend: every step
    converges, new grids nest inside their parents' interiors and cover the
    buffered flags of the level below."""
    hier = amr.build(32, [], eps=0.02, dt=5e-5, qerrortol=1e-9, field="drop")
    prm = amr.RegridParams(maxlevel=2, qtolerance=[0.05, 0.05], ibuffer=[1, 1],
                           desfill=[0.7, 0.7], mgp=[4, 4])
    b = oracle.OracleBackend(2, hier.dt, hier.eps, hier.qerrortol)
    try:
        run = amr.RegridRun(b, hier, prm)
        for _ in range(3):
            nv, res = run.step()
            assert nv < 20 and res < 1e-9
            levels = {d["level"] for d in run.descs}
            assert max(levels) == 2
            for d in run.descs:
                if d["level"] < 1:
                    continue
                p = run.descs[d["parent"]]
                assert p["level"] == d["level"] - 1
                for k in range(2):
                    lo, hi = d["mbounds"][k]
                    assert 1 <= lo <= hi <= p["mx"][k]
                    assert d["mglobal"][k] == [(p["mglobal"][k][0] + lo - 2) * 2 + 1,
                                               (p["mglobal"][k][0] + hi - 1) * 2]
    finally:
        b.close()


def test_after_step_stats_oracle(oracle):
    """The oracle's AfterStepStatistics: on the root alone it is h^2 sum(c)
    and Energy2D; a refined patch holding its parent's values cell by cell
    (piecewise constant) adds no mass."""
    hier = amr.build(16, [(1, (9, 9), (8, 6))], eps=0.05, dt=5e-5, field="drop")
    b = oracle.OracleBackend(2, hier.dt, hier.eps, hier.qerrortol)
    try:
        b.set_hierarchy(hier.descs)
        for p, q in zip(hier.state_patches(), hier.q0s):
            b.put_q(p, q)
        b.set_ghost_level(0)
        root = [i for i, d in enumerate(hier.descs) if d["level"] == 0][0]
        fine = [i for i, d in enumerate(hier.descs) if d["level"] == 1][0]
        qr = b.get_q(root)
        d = hier.descs[fine]
        sl = tuple(slice(d["mbounds"][k][0], d["mbounds"][k][1] + 1) for k in range(2))
        qf = np.zeros_like(b.get_q(fine))
        qf[1:-1, 1:-1, :] = np.kron(qr[sl + (slice(None),)].transpose(2, 0, 1),
                                    np.ones((2, 2))).transpose(1, 2, 0)
        b.put_q(fine, qf)
        b.set_ghost_level(1)
        m, e = b.after_step_stats()
        h = hier.descs[root]["dx"]
        assert m == pytest.approx(h * h * qr[1:-1, 1:-1, 0].sum(), rel=1e-13)
        # Energy: finest level first, Energy2D(fine, h/2) - Energy2D(parent
        # footprint with its ring, h), then the root's Energy2D.
        e_root = oracle.energy2d(h, 1.0, hier.eps, qr[..., 0])
        e_fine = oracle.energy2d(h / 2, 1.0, hier.eps, b.get_q(fine)[..., 0])
        ring = tuple(slice(d["mbounds"][k][0] - 1, d["mbounds"][k][1] + 2) for k in range(2))
        e_foot = oracle.energy2d(h, 1.0, hier.eps, qr[ring + (0,)])
        assert e == pytest.approx((e_fine - e_foot) + e_root, rel=1e-13)
    finally:
        b.close()


def test_served_stream_draws_refined_levels():
    """The served workload gives 2D requests 0, 1 or 2 refined levels and 3D
    requests none, reproducibly."""
    from bsam_b200 import workloads as W
    a = W.config5(200, 100.0)
    b = W.config5(200, 100.0)
    assert [p.maxlevel for _, p in a] == [p.maxlevel for _, p in b]
    lv2 = {p.maxlevel for _, p in a if p.ndims == 2}
    assert lv2 == {0, 1, 2}
    assert all(p.maxlevel == 0 for _, p in a if p.ndims == 3)
    prm = amr.request_params(128, 0.01, 2)
    assert prm.qtolerance == [0.5 / 128 / 0.01, 0.5 / 256 / 0.01]


@pytest.mark.parametrize("n", [0, 1, 2])
def test_buffer_flags_match_reference(gpu_free_lib, n):
    """bsam_host_buffer_flags against BufferAndList + InflateEdgeTags run from
    the reference's own source (tests/golden/ref_buffer_*.npz)."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_golden_reference import _buffer_fixture
    nd, ib, descs, fin, fout = _buffer_fixture(n)
    got = amr.buffer_flags(nd, descs, [f.astype(np.uint8) for f in fin], ib)
    for g, w in zip(got, fout):
        assert np.array_equal(g.astype(np.int64), w)


@pytest.mark.parametrize("n", [0, 1, 2, 3])
def test_new_subgrids_from_summed_area_table_match_reference(gpu_free_lib, n):
    # The clustering that counts from a summed-area table (the form the
    # native AMR driver uses with the device's tables) makes the reference's
    # boxes too.
    d = np.load(os.path.join(GOLD, f"ref_subgrids_{n}.npz"))
    nd = int(d["ndims"])
    got = amr.new_subgrids_sat(amr.summed_area(d["flags"]), float(d["fill"]), int(d["mgp"]))
    assert np.array_equal(got[:, :nd, :], d["boxes"][:, :nd, :])


@pytest.mark.parametrize("seed", [4, 5, 6])
@pytest.mark.parametrize("nd", [2, 3])
def test_new_subgrids_sat_equals_flags(gpu_free_lib, nd, seed):
    rng = np.random.default_rng(seed)
    shape = (40, 36) if nd == 2 else (20, 18, 16)
    fl = (rng.random(shape) < 0.05).astype(np.uint8)
    fl[tuple(slice(3, 9) for _ in range(nd))] = 1
    for fill, mgp in ((0.85, 4), (0.6, 2), (0.95, 3)):
        a = amr.new_subgrids(fl, fill, mgp)
        b = amr.new_subgrids_sat(amr.summed_area(fl), fill, mgp)
        assert np.array_equal(a, b), (fill, mgp)
