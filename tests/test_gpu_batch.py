"""Batched engine (include/bsam_batch.h) on the GPU.

Bars:
  * every problem of a batch gives bit for bit the single-problem library's
    result in the same precision form (final q, V-cycles and residual of
    every time step) -- so a result is the same alone and in any mix;
  * the mixed form stays within 1e-7 of the FP64 oracle;
  * admission follows the pool: a problem that does not fit is refused and
    admitted once a collect frees memory; problems submitted while others run
    give the same results as when solved alone.
"""
import numpy as np
import pytest

import bsam_b200 as B
from bsam_b200 import batch as BB
from bsam_b200 import workloads as W

pytestmark = pytest.mark.gpu


def make(n, seed, nsteps=3, eps=0.01, ndims=2, mean=0.0, tol=1e-8):
    cells = n ** ndims
    u = W.uniform(seed, cells, -1.0, 1.0)
    mx = (n, n, n if ndims == 3 else 1)
    return W.Problem(ndims=ndims, mx=mx, eps=eps, dt=1e-4, nsteps=nsteps, qerrortol=tol,
                     c0=0.5 + 0.5 * mean + 0.025 * u)


def single(prob, precision):
    """The single-problem library with the batch's bottom-kernel size."""
    with B.Solver(prob, precision=precision, bottom_cells=BB.BOTTOM_CELLS) as s:
        r = s.run(prob.nsteps)
    return r


def same(a, b):
    """Batch result a equals single-problem result b bit for bit."""
    assert np.array_equal(a["q"], b["q"][-1]), float(np.max(np.abs(a["q"] - b["q"][-1])))
    assert np.array_equal(a["nvcycles"], b["nvcycles"]), (a["nvcycles"], b["nvcycles"])
    assert np.array_equal(a["residual"], b["residual"]), (a["residual"], b["residual"])
    assert np.array_equal(a["converged"], b["converged"])


MIX2D = [(48, 11, 0.012), (96, 12, 0.008), (128, 13, 0.015), (64, 14, 0.02)]


@pytest.mark.parametrize("precision", [BB.PREC_FP64, BB.PREC_MIXED])
def test_batch_matches_single_solver_2d(gpu_lib, precision):
    probs = [make(n, s, eps=e) for n, s, e in MIX2D]
    got = BB.solve_all(probs, precision=precision)
    for p, g in zip(probs, got):
        same(g, single(p, precision))


@pytest.mark.parametrize("precision", [BB.PREC_FP64, BB.PREC_MIXED])
def test_batch_matches_single_solver_3d(gpu_lib, precision):
    probs = [make(16, 21, nsteps=2, eps=0.03, ndims=3), make(32, 22, nsteps=2, eps=0.02, ndims=3)]
    got = BB.solve_all(probs, precision=precision)
    for p, g in zip(probs, got):
        same(g, single(p, precision))


def test_batch_alone_equals_in_mix(gpu_lib):
    target = make(128, 31, nsteps=4, eps=0.01)
    alone = BB.solve_all([target], precision=BB.PREC_MIXED)[0]
    others = [make(n, 40 + i, nsteps=2 + i % 3, eps=0.005 + 0.003 * i)
              for i, n in enumerate([64, 96, 192, 48, 256])]
    mix = BB.solve_all(others[:2] + [target] + others[2:], precision=BB.PREC_MIXED)[2]
    for k in ("q", "nvcycles", "residual", "converged"):
        assert np.array_equal(alone[k], mix[k]), k
    assert alone["mass"] == mix["mass"]


def test_batch_mixed_against_oracle(gpu_lib, oracle):
    probs = [make(96, 51, nsteps=3, eps=0.01), make(64, 52, nsteps=3, eps=0.015)]
    got = BB.solve_all(probs, precision=BB.PREC_MIXED)
    for p, g in zip(probs, got):
        ref = oracle.run_uniform(p, nsteps=p.nsteps)
        inner = tuple(slice(1, m + 1) for m in p.mx[:p.ndims])
        for v in range(2):
            a, b = g["q"][inner + (v,)], ref["q"][-1][inner + (v,)]
            assert np.max(np.abs(a - b)) / np.max(np.abs(b)) < 1e-7
        assert np.all(g["residual"] < p.qerrortol)
        m0 = p.h ** 2 * p.c0.sum()
        assert abs(g["mass"] - m0) < 10 * p.qerrortol


def test_batch_admission_by_footprint(gpu_lib):
    a, b2 = make(96, 61, nsteps=2), make(96, 62, nsteps=2)
    with BB.Batch(2, precision=BB.PREC_MIXED, max_slots=1) as probe:
        fp = probe.footprint(a)
    assert fp > 0
    with BB.Batch(2, precision=BB.PREC_MIXED, max_slots=4, pool_bytes=fp * 3 // 2) as bt:
        assert bt.footprint(b2) == fp
        sa = bt.submit(a)
        assert sa is not None
        assert bt.submit(b2) is None  # does not fit next to a
        bt.run()
        assert bt.poll() == [sa]
        ra = bt.collect(sa)
        sb = bt.submit(b2)
        assert sb is not None
        bt.run()
        rb = bt.collect(sb)
    same(ra, single(a, BB.PREC_MIXED))
    same(rb, single(b2, BB.PREC_MIXED))


def test_batch_submit_while_running(gpu_lib):
    a, c = make(128, 71, nsteps=4), make(96, 72, nsteps=3)
    with BB.Batch(2, precision=BB.PREC_MIXED, max_slots=4) as bt:
        sa = bt.submit(a)
        for _ in range(60):  # tick until a is past its first time step
            bt.advance(1)
            bt.sync()
            ph, steps = bt.phase(sa)
            if steps > 0:
                break
        assert ph == BB.SLOT_RUNNING and 0 < steps < a.nsteps
        sc = bt.submit(c)  # joins while a is mid-solve
        bt.run()
        assert sorted(bt.poll()) == sorted([sa, sc])
        ra, rc = bt.collect(sa), bt.collect(sc)
    same(ra, single(a, BB.PREC_MIXED))
    same(rc, single(c, BB.PREC_MIXED))


def test_batch_slot_reuse_and_compaction(gpu_lib):
    probs = [make(n, 80 + i, nsteps=1 + i % 3) for i, n in
             enumerate([64, 96, 48, 128, 64, 96, 48, 128, 64, 96, 48, 128])]
    got = BB.solve_all(probs, precision=BB.PREC_MIXED, max_slots=3)
    for p, g in zip(probs, got):
        same(g, single(p, BB.PREC_MIXED))


def test_batch_tuning_leaves_results_unchanged(gpu_lib):
    probs = [make(n, 90 + i) for i, n in enumerate([128, 96, 64])]
    a = BB.solve_all(probs, precision=BB.PREC_MIXED)
    b = BB.solve_all(probs, precision=BB.PREC_MIXED, grid_ctas=7)
    c = BB.solve_all(probs, precision=BB.PREC_MIXED, eager=1)
    d = BB.solve_all(probs, precision=BB.PREC_MIXED, per_pass=1)  # no fused stages
    e = BB.solve_all(probs, precision=BB.PREC_MIXED, fused_ctas=5)
    f = BB.solve_all(probs, precision=BB.PREC_MIXED, tile_chunk=7, fused_chunk=3)
    for x, *others in zip(a, b, c, d, e, f):
        for k in ("q", "nvcycles", "residual"):
            for y in others:
                assert np.array_equal(x[k], y[k]), k


def test_batch_fused_fp64_stage_bit_identical(gpu_lib):
    # FP64 form with the fused shared-memory stage (default) vs per-pass.
    # 160 and 72 leave partial fused tiles (64 x 16 for FP64) at the far edges.
    probs = [make(n, 110 + i, nsteps=2) for i, n in enumerate([192, 160, 72])]
    a = BB.solve_all(probs, precision=BB.PREC_FP64)
    b = BB.solve_all(probs, precision=BB.PREC_FP64, per_pass=1)
    for p, x, y in zip(probs, a, b):
        for k in ("q", "nvcycles", "residual"):
            assert np.array_equal(x[k], y[k]), k
        same(x, single(p, BB.PREC_FP64))


def test_batch_profile_counts_finest_stages(gpu_lib):
    probs = [make(n, 95 + i) for i, n in enumerate([128, 96])]
    with BB.Batch(2, precision=BB.PREC_MIXED, max_slots=2) as bt:
        for p in probs:
            bt.submit(p)
        bt.profile(True)
        bt.advance(2)
        bt.sync()
        st = bt.stats()
        bt.profile(False)
    # two finest-depth stages (pre and post) per tick.  Per cell, FP32
    # working level over an FP32 parent: pre reads f1, f2 and the base (the
    # correction starts from zero), writes the state and restricts q, qs and
    # the base into the parent (5 * 4 / 4); post reads the state, f1, f2, the
    # base and the parent's q and qs (4 * 4 / 4), and reads and writes the
    # FP64 master instead of writing the state
    assert st["smooth_stages"] == 4 and st["smooth_ms"] > 0
    cells = sum(n * n for n in (128, 96))
    pre = 3 * 4 + 2 * 4 + 5
    post = 5 * 4 + 4 + 32
    assert st["smooth_bytes"] == 2 * (pre + post) * cells


def test_submit_many_and_collect_many_match_single_calls(gpu_lib):
    # The batched admission and read-back give the same bits as one call per
    # problem, seeded and from host arrays, page-locked or not; admission
    # stops at the first problem that does not fit.
    probs = [W.seeded(2, n, 0.01, 2, seed=600 + i, cbar=0.5, amp=0.025)
             for i, n in enumerate([64, 96, 128, 48, 192])]
    ref = BB.solve_all(probs, precision=BB.PREC_MIXED)
    with BB.Batch(2, precision=BB.PREC_MIXED, max_slots=8) as bt:
        slots = bt.submit_many(probs)
        assert None not in slots and len(set(slots)) == len(slots)
        bt.run()
        got = bt.collect_many(slots, want_mass=True)
        q0s = [p.q0() for p in probs]
        slots = bt.submit_many(probs, q0s)
        bt.run()
        got2 = bt.collect_many(slots)
    for r, g, g2 in zip(ref, got, got2):
        for k in ("q", "nvcycles", "residual", "converged"):
            assert np.array_equal(r[k], g[k]), k
            assert np.array_equal(r[k], g2[k]), k
        assert r["mass"] == g["mass"]
    with BB.Batch(2, precision=BB.PREC_MIXED, max_slots=3) as bt:
        slots = bt.submit_many(probs)
        assert slots[:3] == sorted(slots[:3]) and slots[3:] == [None, None]
        bt.run()
        got = bt.collect_many(slots[:3])
    for r, g in zip(ref[:3], got):
        assert np.array_equal(r["q"], g["q"])


@pytest.mark.parametrize("nd", [2, 3])
def test_submit_many_from_host_while_a_batch_runs(gpu_lib, nd):
    # Host q0s go through the engine's transfer buffer (one contiguous copy
    # per problem, rows spread into the pitched fields on the device) and
    # results come back the same way, ghost rings included; a second group
    # submitted and advanced while the first solves, and the first collected
    # while the second solves, give the bits of one-at-a-time solves.
    sides = [64, 96, 128, 48] if nd == 2 else [16, 24, 32, 20]
    probs = [W.seeded(nd, n, 0.02 if nd == 3 else 0.01, 2, seed=700 + i, cbar=0.5, amp=0.025)
             for i, n in enumerate(sides)]
    ref = BB.solve_all(probs, precision=BB.PREC_MIXED)
    q0s = [p.q0() for p in probs]
    with BB.Batch(nd, precision=BB.PREC_MIXED, max_slots=2 * len(probs)) as bt:
        a = bt.submit_many(probs, q0s)
        bt.advance(1 << 20)
        b = bt.submit_many(probs[::-1], q0s[::-1])
        bt.advance(1 << 20)
        outs = [np.zeros(q.shape, order="F") for q in q0s]
        got_a = bt.collect_many(a, outs=outs)  # while the second group solves
        got_b = bt.collect_many(b)[::-1]
    for r, g, g2, o in zip(ref, got_a, got_b, outs):
        for k in ("q", "nvcycles", "residual", "converged"):
            assert np.array_equal(r[k], g[k]), k
            assert np.array_equal(r[k], g2[k]), k
        assert g["q"] is o
