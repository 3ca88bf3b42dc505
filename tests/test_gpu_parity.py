"""FP64 parity of the CUDA path (through the C ABI) with the CPU oracle.

Bar (FP64 form): per time step, phi and mu within 1e-11 relative (max norm)
of the oracle, the same V-cycle count, and residuals within 1e-9 relative
(the norm's summation order differs: the GPU reduces in a fixed tree).
"""
import numpy as np
import pytest

import bsam_b200 as B
from bsam_b200 import workloads as W

pytestmark = pytest.mark.gpu

RTOL = 1e-11


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def compare(oracle, prob, nsteps):
    ref = oracle.run_uniform(prob, nsteps=nsteps)
    with B.Solver(prob) as s:
        got = s.run(nsteps)
    inner = tuple(slice(1, m + 1) for m in prob.mx[:prob.ndims])
    for st in range(nsteps):
        for v in range(2):
            e = relerr(got["q"][st][inner + (v,)], ref["q"][st][inner + (v,)])
            assert e <= RTOL, (st, v, e)
        # the ghost ring too (SetGhost semantics incl. edges and corners)
        e = relerr(got["q"][st], ref["q"][st])
        assert e <= RTOL, (st, "ring", e)
    assert np.array_equal(got["nvcycles"], ref["nvcycles"]), (got["nvcycles"], ref["nvcycles"])
    np.testing.assert_allclose(got["residual"], ref["residual"], rtol=1e-9)
    np.testing.assert_allclose(got["mass"], ref["mass"], rtol=1e-13)
    return got, ref


def test_config1_small(gpu_lib, oracle):
    got, ref = compare(oracle, W.config1(nsteps=4, n=32), 4)
    # same arithmetic in the same order: expect bit-identical fields
    assert np.array_equal(got["q"], ref["q"])


def test_config1_full(gpu_lib, oracle):
    compare(oracle, W.config1(nsteps=20), 20)


def test_odd_coarsest_96(gpu_lib, oracle):
    compare(oracle, W.config1(nsteps=3, n=96), 3)


def test_3d_small(gpu_lib, oracle):
    got, ref = compare(oracle, W.config3(nsteps=2, n=32), 2)
    assert np.array_equal(got["q"], ref["q"])


def test_3d_64(gpu_lib, oracle):
    compare(oracle, W.config3(nsteps=2, n=64), 2)


def test_user_bc_2d(gpu_lib, oracle):
    prob = W.config1(nsteps=3, n=64)
    prob.mthbc = (10, 10, 12, 11, 1, 1)
    compare(oracle, prob, 3)


def test_user_bc_3d(gpu_lib, oracle):
    prob = W.config3(nsteps=2, n=16)
    prob.mthbc = (10, 1, 1, 10, 10, 1)
    compare(oracle, prob, 2)


def test_rectangular_2d(gpu_lib, oracle):
    # 128 x 64 root (the shipped example's shape), explicit minlevel = -5.
    prob = W.config1(nsteps=2, n=64)
    prob.mx = (128, 64, 1)
    prob.xupper = (1.0, 0.5, 1.0)
    prob.c0 = 0.5 + 0.025 * W.uniform(11, 128 * 64, -1.0, 1.0)
    prob.minlevel = -5
    compare(oracle, prob, 2)


def test_residual_trace_matches(gpu_lib, oracle):
    prob = W.config1(nsteps=1, n=64)
    ref = oracle.run_uniform(prob, nsteps=1)
    with B.Solver(prob) as s:
        s.step()
        tr = s.trace()
    want = ref["trace"][0][: len(tr)]
    np.testing.assert_allclose(tr, want, rtol=1e-9)


@pytest.mark.parametrize("nd", [2, 3])
def test_put_get_roundtrip(gpu_lib, nd):
    prob = W.config3(nsteps=1, n=8) if nd == 3 else W.config1(nsteps=1, n=12)
    rng = np.random.default_rng(nd)
    with B.Solver(prob) as s:
        q = np.asfortranarray(rng.standard_normal(s.qshape))
        s.put_q(q)
        assert np.array_equal(s.get_q(), q)


# ---- fused smoothing stages (one launch per LevelRelax) ---------------------

def compare_tuned(oracle, prob, nsteps, **tuning):
    ref = oracle.run_uniform(prob, nsteps=nsteps)
    with B.Solver(prob, **tuning) as s:
        got = s.run(nsteps)
    assert np.array_equal(got["nvcycles"], ref["nvcycles"])
    for st in range(nsteps):
        e = relerr(got["q"][st], ref["q"][st])
        assert e <= RTOL, (st, e)
    return got, ref


@pytest.mark.parametrize("chunk", [0, 5, 64])
def test_fused_3d_bit_identical(gpu_lib, oracle, chunk):
    # 48^3: levels 48, 24, 12 fused (several tiles, partial tiles, chunks with
    # a remainder), 6 and 3 on the per-pass path.
    prob = W.config3(nsteps=2, n=48)
    got, ref = compare_tuned(oracle, prob, 2, fuse=1, fuse_min_n=8, chunk=chunk)
    assert np.array_equal(got["q"], ref["q"])


def test_fused_3d_rectangular_userbc(gpu_lib, oracle):
    prob = W.config3(nsteps=2, n=32)
    prob.mx = (64, 32, 48)
    prob.xupper = (1.0, 0.5, 0.75)
    prob.c0 = 0.55 + 0.025 * W.uniform(31, 64 * 32 * 48, -1.0, 1.0)
    prob.mthbc = (10, 1, 1, 10, 1, 10)
    got, ref = compare_tuned(oracle, prob, 2, fuse=1, fuse_min_n=8, chunk=7)
    assert np.array_equal(got["q"], ref["q"])


def test_fused_matches_unfused_128(gpu_lib):
    prob = W.config3(nsteps=1, n=128)
    with B.Solver(prob, fuse=0) as a:
        ra = a.run(1)
    with B.Solver(prob, fuse=1) as b:
        rb = b.run(1)
    assert np.array_equal(ra["q"], rb["q"]) and np.array_equal(ra["nvcycles"], rb["nvcycles"])


@pytest.mark.parametrize("nd,n", [(2, 128), (2, 96), (3, 32)])
def test_bottom_kernel_matches_per_level_launches(gpu_lib, nd, n):
    # The single-CTA bottom of the V-cycle (levels <= 4096 cells) against one
    # launch per phase: the same arithmetic, so bit-identical fields.
    prob = W.config1(nsteps=2, n=n) if nd == 2 else W.config3(nsteps=2, n=n)
    with B.Solver(prob, bottom_cells=-1) as a:
        ra = a.run(2)
    with B.Solver(prob) as b:
        rb = b.run(2)
    assert np.array_equal(ra["q"], rb["q"]) and np.array_equal(ra["nvcycles"], rb["nvcycles"])


@pytest.mark.parametrize("nd,n", [(2, 256), (3, 64)])
def test_graph_loop_matches_host_loop(gpu_lib, nd, n):
    # The device-side WHILE loop of the step graph stops after the same
    # V-cycle as the host loop and leaves identical fields and residuals.
    prob = W.config1(nsteps=3, n=n) if nd == 2 else W.config3(nsteps=2, n=n)
    with B.Solver(prob, graph=-1) as a:
        ra = a.run(prob.nsteps)
        ta = a.trace()
    with B.Solver(prob) as b:
        rb = b.run(prob.nsteps)
        tb = b.trace()
    assert np.array_equal(ra["q"], rb["q"])
    assert np.array_equal(ra["nvcycles"], rb["nvcycles"])
    assert np.array_equal(ra["residual"], rb["residual"]) and np.array_equal(ta, tb)


def test_energy_matches_oracle_and_decays(gpu_lib, oracle):
    # Energy2D of the root state (AfterStep2D, level 0) on the device against
    # the oracle's sequential sums, after every step; Eyre's splitting makes
    # it non-increasing.
    prob = W.config1(nsteps=4, n=64)
    with B.Solver(prob) as s:
        e = [s.energy()]
        assert abs(e[0] - oracle.energy2d(prob.h, prob.alpha, prob.eps, s.get_q()[..., 0])) <= (
            1e-12 * abs(e[0]))
        for _ in range(4):
            s.step()
            q = s.get_q()
            e.append(s.energy())
            want = oracle.energy2d(prob.h, prob.alpha, prob.eps, q[..., 0])
            assert abs(e[-1] - want) <= 1e-12 * abs(want), (e[-1], want)
    assert all(b <= a for a, b in zip(e, e[1:])), e


def test_energy_unsupported_in_3d(gpu_lib):
    with B.Solver(W.config3(nsteps=1, n=16)) as s:
        with pytest.raises(B.BsamError):
            s.energy()


@pytest.mark.parametrize("n", [64, 128])
def test_periodic_shipped_example_codes(gpu_lib, oracle, n):
    # The shipped example's faces (griddata.dat:61-66: periodic x, user code
    # 10 on y) and its eps and dt (problemdata.dat, rundata.dat) on an
    # n x n/2 root over [0, 12.8] x [0, 6.4], seeded initial state, no
    # refined levels.
    prob = W.config1(nsteps=3, n=n)
    prob.mx = (n, n // 2, 1)
    prob.xupper = (12.8, 6.4, 1.0)
    prob.mthbc = (2, 2, 10, 10, 1, 1)
    prob.eps, prob.dt, prob.qerrortol = 0.018, 0.1, 1e-8
    prob.c0 = 0.5 + 0.025 * W.uniform(41, n * (n // 2), -1.0, 1.0)
    got, ref = compare(oracle, prob, 3)
    assert np.array_equal(got["q"], ref["q"])


def test_periodic_3d_and_mixed(gpu_lib, oracle):
    prob = W.config3(nsteps=2, n=32)
    prob.mthbc = (2, 2, 1, 1, 2, 2)
    compare(oracle, prob, 2)
    prob.qerrortol = 1e-8
    ref = oracle.run_uniform(prob, nsteps=2)
    with B.Solver(prob, precision=B.PREC_MIXED) as s:
        got = s.run(2)
    for st in range(2):
        assert relerr(got["q"][st], ref["q"][st]) < 1e-7
    assert np.all(got["residual"] < prob.qerrortol)


def test_periodic_rejections(gpu_lib):
    prob = W.config1(nsteps=1, n=96)   # periodic extent 96 -> ... -> 3 (odd, above 1)
    prob.mthbc = (2, 2, 1, 1, 1, 1)
    with pytest.raises(B.BsamError):
        B.Solver(prob)
    prob = W.config1(nsteps=1, n=64)   # an unpaired periodic face
    prob.mthbc = (2, 1, 1, 1, 1, 1)
    with pytest.raises(B.BsamError):
        B.Solver(prob)
