"""The allocation-free residual norm entry point, through the C ABI.

bsam_gpu_resid_norm_noalloc serves callers that cannot allocate device memory
when they need the norm (their device memory belongs to their own pool, or
their step loop must not take cudaMalloc's implicit synchronisation).  Its
scratch is a fixed array compiled into the library.  This file is collected
last so that a run stopping at the first failure has run every other test.
"""
import ctypes

import numpy as np
import pytest

import bsam_b200 as B
from bsam_b200 import workloads as W

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _dev_ptr(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("nd", [2, 3])
def test_noalloc_matches_multigrid_residual_twice(gpu_lib, nd):
    import torch
    prob = W.config1(nsteps=1, n=64) if nd == 2 else W.config3(nsteps=1, n=32)
    with B.Solver(prob) as s:
        nv, res, conv = s.step()
        q = s.get_q()
        f = s.get_f()
        dx = s.patches[0].dx
    # The caller owns its inputs and outputs; the entry point allocates nothing.
    qd = torch.from_numpy(q.ravel(order="F").copy()).cuda()
    fd = torch.from_numpy(f.ravel(order="F").copy()).cuda()
    mx = (ctypes.c_int32 * 3)(*[prob.mx[d] if d < nd else 1 for d in range(3)])
    stream = torch.cuda.current_stream()
    for call in range(2):
        out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
        rc = gpu_lib.bsam_gpu_resid_norm_noalloc(
            torch.cuda.current_device(), nd, mx, dx, prob.dt, prob.eps, prob.alpha,
            _dev_ptr(qd), _dev_ptr(fd), _dev_ptr(out), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, gpu_lib.bsam_gpu_strerror(rc)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_allclose(got[0], res, rtol=RTOL, err_msg=f"call {call}")
        denom = 2.0 * np.prod(prob.mx[:nd])
        np.testing.assert_allclose(got[1], res * res * denom, rtol=1e-10, err_msg=f"call {call}")


@pytest.mark.parametrize("nd,mx", [(2, (130, 37)), (3, (70, 9, 5))])
def test_noalloc_ragged_tiles_against_oracle_operator(gpu_lib, oracle, nd, mx):
    # Several tiles in x with a partial last one, and a partial last tile in
    # y: known q (ring included) and f, the residual norm of f - Operator(q)
    # with the oracle's Operator, on two calls in a row.
    import torch
    rng = np.random.default_rng(7 + nd)
    qshape = tuple(m + 2 for m in mx) + (2,)
    q = np.asfortranarray(0.5 + 0.1 * rng.standard_normal(qshape))
    f = np.asfortranarray(0.01 * rng.standard_normal(tuple(mx) + (2,)))
    h, dt, eps, alpha = 1.0 / mx[0], 1e-4, 0.02, 1.0
    rf = f - oracle.operator(nd, mx, h, dt, alpha, eps, q)
    total = float(np.sum(rf * rf))
    denom = 2.0 * np.prod(mx)
    qd = torch.from_numpy(q.ravel(order="F").copy()).cuda()
    fd = torch.from_numpy(f.ravel(order="F").copy()).cuda()
    m = (ctypes.c_int32 * 3)(*(list(mx) + [1] * (3 - nd)))
    stream = torch.cuda.current_stream()
    for call in range(2):
        out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
        rc = gpu_lib.bsam_gpu_resid_norm_noalloc(
            torch.cuda.current_device(), nd, m, h, dt, eps, alpha, _dev_ptr(qd), _dev_ptr(fd),
            _dev_ptr(out), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, gpu_lib.bsam_gpu_strerror(rc)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_allclose(got[1], total, rtol=RTOL, err_msg=f"call {call}")
        np.testing.assert_allclose(got[0], np.sqrt(total / denom), rtol=RTOL)
        np.testing.assert_allclose(got[1] / denom, got[0] ** 2, rtol=1e-12)


def test_noalloc_rejects_patch_beyond_scratch(gpu_lib):
    mx = (ctypes.c_int32 * 3)(4096, 4100, 1)   # 64 x 1025 tiles > 65536
    null = ctypes.c_void_p(16)
    rc = gpu_lib.bsam_gpu_resid_norm_noalloc(0, 2, mx, 1.0 / 4096, 1e-4, 0.01, 1.0,
                                             null, null, null, None)
    assert rc == -8
    assert b"static scratch" in gpu_lib.bsam_gpu_strerror(rc)
