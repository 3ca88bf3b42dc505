"""Host logic of the served form (no GPU): the request stream of the serving
workload, the regrid settings a refined request gets, and the latency and
throughput summary the bench line reports."""
import numpy as np
import pytest

from bsam_b200 import amr
from bsam_b200 import serve as SV
from bsam_b200 import workloads as W


def test_config5_stream_shape():
    reqs = W.config5(600, 500.0)
    arrivals = np.array([a for a, _ in reqs])
    assert np.all(np.diff(arrivals) > 0)
    # Poisson arrivals: mean gap about 1 / rate.
    assert abs(np.mean(np.diff(arrivals)) - 1.0 / 500.0) < 0.25 / 500.0
    probs = [p for _, p in reqs]
    nd3 = [p for p in probs if p.ndims == 3]
    assert 0.2 < len(nd3) / len(probs) < 0.4
    assert {int(p.mx[0]) for p in nd3} <= {32, 64, 128}
    p2 = [p for p in probs if p.ndims == 2]
    assert {int(p.mx[0]) for p in p2} <= {64, 128, 256, 512}
    levels = [p.maxlevel for p in p2]
    assert set(levels) == {0, 1, 2}
    assert all(getattr(p, "maxlevel", 0) == 0 for p in nd3)
    assert all(1 <= p.nsteps <= 50 for p in probs)
    assert all(0.005 <= p.eps <= 0.02 for p in probs)
    # The same stream at every rate: only the arrival times scale.
    other = W.config5(600, 1000.0)
    assert [(p.ndims, int(p.mx[0]), p.nsteps) for _, p in other] == \
        [(p.ndims, int(p.mx[0]), p.nsteps) for p in probs]
    assert np.allclose([a for a, _ in other], arrivals / 2.0)


@pytest.mark.parametrize("n,eps,maxlevel", [(64, 0.01, 1), (256, 0.005, 2)])
def test_request_regrid_settings(n, eps, maxlevel):
    prm = amr.request_params(n, eps, maxlevel)
    assert prm.maxlevel == maxlevel
    # |grad phi| > 0.5/eps on the undivided gradient: 0.5 h / eps per level.
    for level in range(maxlevel):
        h = 1.0 / (n * 2 ** level)
        assert prm.qtolerance[level] == pytest.approx(0.5 * h / eps)
    assert prm.ibuffer == [1] * maxlevel and prm.mgp == [8] * maxlevel
    assert prm.desfill == [0.9] * maxlevel


def _req(rid, arrival, latency, maxlevel, nsteps=3, nv=(4, 5, 6), conv=1):
    p = W.seeded(2, 64, 0.01, nsteps, seed=rid, cbar=0.5, amp=0.025)
    p.maxlevel = maxlevel
    r = SV.Request(rid, arrival, p)
    r.admitted = arrival
    r.finished = arrival + latency
    r.result = {"nvcycles": np.array(nv[:nsteps]), "converged": np.full(nsteps, conv)}
    return r


def test_summary_latency_split_and_rates():
    lat_u = [0.010, 0.020, 0.030, 0.040]
    lat_a = [0.100, 0.300]
    reqs = [_req(i, 0.01 * i, l, 0) for i, l in enumerate(lat_u)]
    reqs += [_req(10 + i, 0.05 + 0.01 * i, l, 1 + i) for i, l in enumerate(lat_a)]
    s = SV.summarize(reqs)
    assert s["requests"] == 6 and s["amr_requests"] == 2
    assert s["uniform_p50_ms"] == pytest.approx(1e3 * np.percentile(lat_u, 50))
    assert s["amr_p50_ms"] == pytest.approx(1e3 * np.percentile(lat_a, 50))
    assert s["p99_ms"] == pytest.approx(1e3 * np.percentile(lat_u + lat_a, 99))
    makespan = max(r.finished for r in reqs) - min(r.arrival for r in reqs)
    assert s["makespan_s"] == pytest.approx(makespan)
    assert s["solves_per_s"] == pytest.approx(6 / makespan)
    assert s["steps_per_s"] == pytest.approx(18 / makespan)
    assert s["vcycles"] == 6 * 15
    assert s["all_converged"]
    reqs.append(_req(20, 0.2, 0.05, 0, conv=0))
    assert not SV.summarize(reqs)["all_converged"]
