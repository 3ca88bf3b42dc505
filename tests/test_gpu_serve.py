"""Served form (bsam_b200/serve.py) on the GPU.

Bars: a request's result is bit-identical whether it is solved alone or
admitted into a running mix of other requests; requests that arrive while
others run are admitted into the running batch (their work overlaps); when
the pool is full, requests wait and are admitted as memory frees up; the
device-side initial state equals the host-built one bit for bit.
"""
import numpy as np
import pytest

from bsam_b200 import batch as BB
from bsam_b200 import serve as SV
from bsam_b200 import workloads as W

pytestmark = pytest.mark.gpu


def small_stream(nreq, rate, seed=3):
    rng_sides2 = (64, 96, 128)
    rng_sides3 = (16, 32)
    stream, t = [], 0.0
    gaps = -np.log(1.0 - W.uniform(seed, nreq, 0.0, 1.0)) / rate
    for r in range(nreq):
        t += float(gaps[r])
        if r % 3 == 2:
            n, nd = rng_sides3[r % 2], 3
        else:
            n, nd = rng_sides2[r % 3], 2
        p = W.seeded(nd, n, eps=0.008 + 0.001 * (r % 5), nsteps=2 + r % 3, seed=1000 + r,
                     cbar=0.5, amp=0.025)
        stream.append((t, p))
    return stream


def alone(prob):
    with BB.Batch(prob.ndims, precision=BB.PREC_MIXED, max_slots=1) as b:
        s = b.submit_seeded(prob)
        b.run()
        return b.collect(s)


@pytest.mark.parametrize("nd,n", [(2, 96), (3, 32)])
def test_seeded_state_equals_host_state(gpu_lib, nd, n):
    p = W.seeded(nd, n, eps=0.01, nsteps=2, seed=77, cbar=0.5, amp=0.025)
    with BB.Batch(nd, precision=BB.PREC_MIXED, max_slots=2) as b:
        s1 = b.submit_seeded(p)
        s2 = b.submit(p, p.q0())
        b.run()
        r1, r2 = b.collect(s1), b.collect(s2)
    for k in ("q", "nvcycles", "residual"):
        assert np.array_equal(r1[k], r2[k]), k


def test_serve_same_alone_and_in_mix(gpu_lib):
    stream = small_stream(18, rate=3000.0)
    with SV.Server(pool_bytes=2 << 30, max_slots=32, ticks=2, keep_q=True) as srv:
        reqs = srv.serve(stream)
    summ = SV.summarize(reqs)
    assert summ["all_converged"], summ
    # Work overlapped: some request was admitted before an earlier one finished.
    overlap = any(b.admitted < a.finished for a in reqs for b in reqs if b.rid > a.rid)
    assert overlap
    for r in (reqs[0], reqs[5], reqs[8]):
        ref = alone(r.prob)
        for k in ("q", "nvcycles", "residual", "converged"):
            assert np.array_equal(r.result[k], ref[k]), (r.rid, k)


def test_serve_admission_waits_for_memory(gpu_lib):
    stream = small_stream(10, rate=5000.0, seed=9)
    # Pool for about two of the largest 2D requests at a time per engine.
    with BB.Batch(2, precision=BB.PREC_MIXED, max_slots=1) as probe:
        big = max(probe.footprint(p) for _, p in stream if p.ndims == 2)
    with SV.Server(pool_bytes=4 * big + (64 << 20), max_slots=8, ticks=2) as srv:
        reqs = srv.serve(stream)
    assert all(r.result is not None for r in reqs)
    waited = [r for r in reqs if r.admitted - r.arrival > 1e-4]
    assert waited, "expected some requests to wait for pool memory"
    assert SV.summarize(reqs)["all_converged"]


def test_serve_amr_requests_same_alone(gpu_lib):
    """2D requests with refined levels run in their own batch beside the
    uniform ones (drivers built by worker threads, V-cycles in shared
    launches, regridded between steps): each result equals the same request
    solved alone by its native driver, bit for bit, and the batch requests of
    the mix still converge."""
    stream = small_stream(8, rate=3000.0)
    amr_ids = (1, 4, 6)
    for rid in amr_ids:
        p = stream[rid][1]
        p.maxlevel = 1 + rid % 2
        p.nsteps = 3
    with SV.Server(pool_bytes=2 << 30, max_slots=32, ticks=2, keep_q=True,
                   amr_workers=2) as srv:
        reqs = srv.serve(stream)
    summ = SV.summarize(reqs)
    assert summ["all_converged"] and summ["amr_requests"] == len(amr_ids), summ
    from bsam_b200 import amr
    for rid in amr_ids:
        r = reqs[rid]
        ref = amr.solve_request(r.prob, keep_q=True)
        for k in ("nvcycles", "residual", "converged"):
            assert np.array_equal(r.result[k], ref[k]), (rid, k)
        assert r.result["descs"] == ref["descs"]
        for (i, q), (j, qr) in zip(r.result["q"], ref["q"]):
            assert i == j and np.array_equal(q, qr), (rid, i)
