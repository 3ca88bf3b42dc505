"""Refined (AMR) hierarchies in the batched engine (bsam_batch_submit_amr).

Bar: the time steps of a refined problem run inside a batch give, bit for
bit, what its native AMR driver gives stepping alone (bsam_amr_step): the
same grids after every regrid, the same V-cycle counts and residuals, the
same q on every patch -- alone in a batch, beside other refined problems,
and beside uniform problems of the mixed form, whose own results do not
change either.
"""
import numpy as np
import pytest

from bsam_b200 import amr
from bsam_b200 import batch as BB
from bsam_b200 import workloads as W

pytestmark = pytest.mark.gpu

PARAMS = {
    # ndims: (eps, RegridParams) -- the regrid tests' settings
    2: (0.02, amr.RegridParams(maxlevel=2, qtolerance=[0.05, 0.05], ibuffer=[1, 1],
                               desfill=[0.7, 0.7], mgp=[4, 4])),
    3: (0.05, amr.RegridParams(maxlevel=2, qtolerance=[0.15, 0.15], ibuffer=[1, 1],
                               desfill=[0.7, 0.7], mgp=[2, 2])),
}


def case(n, seed, nd=2):
    eps, prm = PARAMS[nd]
    hier = amr.build(n, [], eps=eps, dt=5e-5, qerrortol=1e-9, field="drop", ndims=nd, seed=seed)
    return hier, prm


def alone(hier, prm, nsteps):
    """The native driver stepping by itself."""
    with amr.AmrRun(hier, prm) as r:
        nv, res, grids = [], [], []
        for _ in range(nsteps):
            a, b = r.step()
            nv.append(a)
            res.append(b)
            grids.append(len(r.descs))
        return {"nvcycles": np.array(nv), "residual": np.array(res), "descs": r.descs,
                "q": r.state(), "patches": grids}


def batched(cases, nsteps, nd=2, precision=BB.PREC_FP64, uniform=()):
    """The same problems' steps in one batch (with uniform problems beside)."""
    runs = []
    try:
        for h, p in cases:
            runs.append(amr.AmrRun(h, p))
        with BB.Batch(nd, precision=precision, max_slots=len(cases) + len(uniform),
                      qerrortol=1e-8, maxvcycles=20) as b:
            slots = [b.submit_amr(r, nsteps) for r in runs]
            assert all(s is not None for s in slots)
            uslots = [b.submit(u) for u in uniform]
            b.run()
            got = [b.collect_amr(s) for s in slots]
            ugot = [b.collect(s) for s in uslots]
        for r, g in zip(runs, got):
            g["descs"] = r.descs
            g["q"] = r.state()
        return got, ugot
    finally:
        for r in runs:
            r.close()


def same(g, a):
    assert g["descs"] == a["descs"]
    assert np.array_equal(g["nvcycles"], a["nvcycles"]), (g["nvcycles"], a["nvcycles"])
    assert np.array_equal(g["residual"], a["residual"]), (g["residual"], a["residual"])
    assert len(g["q"]) == len(a["q"])
    for (i, qg), (j, qa) in zip(g["q"], a["q"]):
        assert i == j
        assert np.array_equal(qg, qa), (i, float(np.max(np.abs(qg - qa))))


@pytest.mark.parametrize("nd,n,nsteps", [(2, 32, 3), (3, 16, 2)])
def test_batch_amr_matches_native_driver(gpu_lib, nd, n, nsteps):
    h, p = case(n, 3, nd)
    a = alone(h, p, nsteps)
    assert max(a["patches"]) > len([d for d in h.descs if d["level"] <= 0]), \
        "the case must refine"
    (g,), _ = batched([case(n, 3, nd)], nsteps, nd)
    same(g, a)


def test_batch_amr_beside_refined_and_uniform_problems(gpu_lib):
    """Three refined problems of different roots in a mixed-precision batch
    with three uniform problems: each refined result equals its driver's
    alone, each uniform result equals the batch's result for it alone."""
    specs = [(32, 5), (48, 6), (64, 7)]
    nsteps = 3
    ref = [alone(*case(n, s), nsteps) for n, s in specs]

    def uni(n, seed, steps):
        u = W.uniform(seed, n * n, -1.0, 1.0)
        return W.Problem(ndims=2, mx=(n, n, 1), eps=0.01, dt=1e-4, nsteps=steps, qerrortol=1e-8,
                         c0=0.5 + 0.025 * u)

    uniform = [uni(64, 51, 2), uni(96, 52, 4), uni(128, 53, 3)]
    ualone = BB.solve_all(uniform, precision=BB.PREC_MIXED)
    got, ugot = batched([case(n, s) for n, s in specs], nsteps, precision=BB.PREC_MIXED,
                        uniform=uniform)
    for g, a in zip(got, ref):
        same(g, a)
    for g, a in zip(ugot, ualone):
        for k in ("q", "nvcycles", "residual", "converged"):
            assert np.array_equal(g[k], a[k]), k


def test_batch_amr_config2_sustained(gpu_lib):
    """The 2D AMR workload (256^2 root, two refined levels, sustained
    refinement: about 140 refined patches) for two problems, two steps."""
    ref, cases = [], []
    for seed in (2, 9):
        h, p = amr.config2(sustained=True, seed=seed)
        ref.append(alone(h, p, 2))
        cases.append(amr.config2(sustained=True, seed=seed))
    got, _ = batched(cases, 2)
    for g, a in zip(got, ref):
        assert max(a["patches"]) > 50
        same(g, a)


def test_batch_amr_table_growth_compaction_and_slot_reuse(gpu_lib):
    """Sixteen problems of the sustained AMR workload for five steps: their
    records outgrow the refined table (reallocation, graph captured again)
    and retired blocks outnumber the live ones (compaction) -- every result
    still equals its driver's alone.  The freed slots then take uniform
    problems of the mixed form, whose results equal their batch alone."""
    nsteps = 5
    seeds = list(range(40, 56))
    ref = [alone(*amr.config2(sustained=True, seed=s), nsteps) for s in seeds]
    runs = [amr.AmrRun(*amr.config2(sustained=True, seed=s)) for s in seeds]
    uni = [W.seeded(2, n, 0.01, 2, seed=700 + n, cbar=0.5, amp=0.025) for n in (64, 96, 128)]
    ualone = BB.solve_all(uni, precision=BB.PREC_MIXED)
    try:
        with BB.Batch(2, precision=BB.PREC_MIXED, max_slots=len(seeds), qerrortol=1e-8,
                      maxvcycles=20) as b:
            slots = [b.submit_amr(r, nsteps) for r in runs]
            b.run()
            got = [b.collect_amr(s) for s in slots]
            st = b.stats()
            assert st["regrids"] == len(seeds) * nsteps
            assert st["captures"] >= 2
            uslots = [b.submit(u) for u in uni]
            assert all(s is not None for s in uslots)
            b.run()
            ugot = [b.collect(s) for s in uslots]
        for r, g, a in zip(runs, got, ref):
            g["descs"] = r.descs
            g["q"] = r.state()
            same(g, a)
        for g, a in zip(ugot, ualone):
            for k in ("q", "nvcycles", "residual", "converged"):
                assert np.array_equal(g[k], a[k]), k
    finally:
        for r in runs:
            r.close()
