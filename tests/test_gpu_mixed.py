"""Mixed precision (FP32 FAS V-cycle inside an FP64 defect-correction loop)
against the FP64 oracle.

Bar: after every time step, phi and mu within 1e-7 (max norm, relative to the
field's max magnitude) of the oracle's FP64 solution, the FP64 residual below
qerrortol, and at most two more V-cycles than the FP64 form needs.
"""
import numpy as np
import pytest

import bsam_b200 as B
from bsam_b200 import workloads as W

pytestmark = pytest.mark.gpu

ERR = 1e-7


def run_mixed(oracle, prob, nsteps, **tuning):
    ref = oracle.run_uniform(prob, nsteps=nsteps)
    with B.Solver(prob, precision=B.PREC_MIXED, **tuning) as s:
        got = s.run(nsteps)
    inner = tuple(slice(1, m + 1) for m in prob.mx[:prob.ndims])
    errs = []
    for st in range(nsteps):
        for v in range(2):
            a, b = got["q"][st][inner + (v,)], ref["q"][st][inner + (v,)]
            e = float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
            errs.append(e)
            assert e < ERR, (st, v, e)
    assert np.all(got["residual"] < prob.qerrortol), got["residual"]
    assert np.all(got["converged"] == 1)
    assert np.all(got["nvcycles"] <= ref["nvcycles"] + 2), (got["nvcycles"], ref["nvcycles"])
    return got, ref, max(errs)


@pytest.mark.parametrize("n", [128, 96])
def test_mixed_2d(gpu_lib, oracle, n):
    prob = W.config1(nsteps=4, n=n)
    prob.qerrortol = 1e-8
    run_mixed(oracle, prob, 4)


def test_mixed_3d(gpu_lib, oracle):
    run_mixed(oracle, W.config3(nsteps=2, n=64), 2)


def test_mixed_3d_fused_fp32_stages(gpu_lib, oracle):
    run_mixed(oracle, W.config3(nsteps=2, n=64), 2, fuse=1, fuse_min_n=16)


def test_mixed_host_loop_matches_graph(gpu_lib):
    prob = W.config1(nsteps=3, n=128)
    prob.qerrortol = 1e-8
    with B.Solver(prob, precision=B.PREC_MIXED, graph=-1) as a:
        ra = a.run(3)
    with B.Solver(prob, precision=B.PREC_MIXED) as b:
        rb = b.run(3)
    assert np.array_equal(ra["q"], rb["q"]) and np.array_equal(ra["nvcycles"], rb["nvcycles"])


def test_mixed_mass_fp64(gpu_lib, oracle):
    prob = W.config1(nsteps=3, n=128)
    prob.qerrortol = 1e-8
    got, ref, _ = run_mixed(oracle, prob, 3)
    m0 = prob.h ** 2 * prob.c0.sum()
    assert np.all(np.abs(got["mass"] - m0) < 10 * prob.qerrortol)


def test_mixed_small_problem_all_fp64_levels(gpu_lib, oracle):
    # 48^2 <= 4096 cells: every level of the inner cycle stays FP64.
    prob = W.config1(nsteps=2, n=48)
    prob.qerrortol = 1e-8
    run_mixed(oracle, prob, 2)
