"""Parity at the benchmark configurations' full sizes, against the oracle.

* 3D 128^3 (eps 0.02, dt 1e-4, off-critical quench), first three time
  steps: the FP64 form within 1e-11 of the oracle after every step with the
  same V-cycle counts; the mixed form within 1e-7 with its FP64 residual
  below qerrortol.
* 2D AMR, a 256^2 root with two refined levels regridded every step (the
  drop, eps 0.005, dt 5e-5), with the configured tag threshold and with the
  sustained one: the native driver takes the oracle's grids, V-cycle counts
  and states (1e-11) step for step.
* The batched mixed form on the largest sides of the 512-problem workload
  (192^2 and 256^2, all ten steps): within 1e-7 of the oracle.
"""
import numpy as np
import pytest

import bsam_b200 as B
from bsam_b200 import amr
from bsam_b200 import batch as BB
from bsam_b200 import workloads as W

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def cfg3_ref(oracle):
    prob = W.config3(nsteps=3)
    return prob, oracle.run_uniform(prob, nsteps=3)


def test_config3_128cubed_fp64(gpu_lib, cfg3_ref):
    prob, ref = cfg3_ref
    with B.Solver(prob) as s:
        got = s.run(3)
    assert np.array_equal(got["nvcycles"], ref["nvcycles"]), (got["nvcycles"], ref["nvcycles"])
    inner = tuple(slice(1, m + 1) for m in prob.mx[:3])
    for st in range(3):
        for v in range(2):
            e = relerr(got["q"][st][inner + (v,)], ref["q"][st][inner + (v,)])
            assert e <= 1e-11, (st, v, e)
        assert relerr(got["q"][st], ref["q"][st]) <= 1e-11
    np.testing.assert_allclose(got["residual"], ref["residual"], rtol=1e-9)


def test_config3_128cubed_mixed(gpu_lib, cfg3_ref):
    prob, ref = cfg3_ref
    with B.Solver(prob, precision=B.PREC_MIXED) as s:
        got = s.run(3)
    inner = tuple(slice(1, m + 1) for m in prob.mx[:3])
    for st in range(3):
        for v in range(2):
            e = relerr(got["q"][st][inner + (v,)], ref["q"][st][inner + (v,)])
            assert e < 1e-7, (st, v, e)
    assert np.all(got["residual"] < prob.qerrortol) and np.all(got["converged"] == 1)
    assert np.all(got["nvcycles"] <= ref["nvcycles"] + 2), (got["nvcycles"], ref["nvcycles"])


@pytest.mark.parametrize("sustained", [False, True])
def test_config2_256sq_two_levels(gpu_lib, oracle, sustained):
    hier, prm = amr.config2(sustained=sustained)
    o = oracle.OracleBackend(2, hier.dt, hier.eps, hier.qerrortol)
    with amr.AmrRun(hier, prm) as rn:
        try:
            ro = amr.RegridRun(o, hier, prm)
            levels = set()
            for step in range(3):
                nvn, _ = rn.step()
                nvo, _ = ro.step()
                assert rn.descs == ro.descs, f"grids differ at step {step}"
                assert nvn == nvo, (step, nvn, nvo)
                levels |= {d["level"] for d in rn.descs}
                for (i, qg), (_, qo) in zip(rn.state(), ro.state()):
                    d = rn.descs[i]
                    inner = tuple(slice(1, m + 1) for m in d["mx"][:2])
                    np.testing.assert_allclose(qg[inner], qo[inner], rtol=0, atol=1e-11)
            assert 2 in levels  # both refined levels were exercised
        finally:
            o.close()


def test_batch_mixed_largest_sides_against_oracle(gpu_lib, oracle):
    work = W.config4(nprob=64, nsteps=10, seed=4)
    probs = [next(p for p in work if p.mx[0] == n) for n in (192, 256)]
    got = BB.solve_all(probs, precision=BB.PREC_MIXED)
    for p, g in zip(probs, got):
        ref = oracle.run_uniform(p, nsteps=p.nsteps, keep_steps=False, final_q=True)
        inner = tuple(slice(1, m + 1) for m in p.mx[:2])
        for v in range(2):
            e = relerr(g["q"][inner + (v,)], ref["q_final"][inner + (v,)])
            assert e < 1e-7, (p.mx[0], v, e)
        assert np.all(g["residual"] < p.qerrortol) and np.all(g["converged"] == 1)
