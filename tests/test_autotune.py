"""The autotuner's search and cache logic on the CPU (fake timings)."""
import dataclasses

from bsam_b200 import autotune as AT
from bsam_b200 import batch as BB
from bsam_b200 import workloads as W


def test_coordinate_descent_finds_separable_optimum():
    # A separable cost with one best value per knob: the descent finds it.
    best = {"per_pass": 0, "fused_occ": 4, "fused_ctas": 3 * 148, "grid_ctas": 8 * 148,
            "tile_chunk": 4, "fused_chunk": 2}
    calls = []

    def timer(c):
        calls.append(c)
        d = c.as_dict()
        return 10.0 + sum(abs(d[k] - best[k]) / (1 + best[k]) for k in AT.KNOBS)

    res = AT.search([], BB.PREC_MIXED, timer=timer, nsm=148)
    assert res["choice"] == best
    assert res["gain"] > 1.0 and res["ms"] <= res["default_ms"]
    assert len(calls) == len(set(calls))  # every candidate timed once
    assert len(res["timings"]) == len(calls)


def test_default_kept_when_nothing_is_faster():
    res = AT.search([], BB.PREC_FP64, timer=lambda c: 5.0, nsm=148)
    assert res["choice"] == AT.Choice().as_dict() and res["gain"] == 1.0


def test_workload_class_and_stratified_sample():
    probs = W.config4(nprob=64, nsteps=10, seed=4)
    assert AT.workload_class(probs) == "2d:64,96,128,192,256"
    s = AT.stratified(probs, 2)
    assert len(s) == 10
    assert sorted({p.mx[0] for p in s}) == [64, 96, 128, 192, 256]


def test_cache_roundtrip(tmp_path):
    path = str(tmp_path / "t.json")
    assert AT.load_cache(path) == {}
    AT.store("k1", {"choice": {"fused_occ": 3}}, path)
    AT.store("k2", {"choice": {"fused_occ": 4}}, path)
    d = AT.load_cache(path)
    assert d["k1"]["choice"]["fused_occ"] == 3 and d["k2"]["choice"]["fused_occ"] == 4


def test_candidates_are_valid_tuning_values():
    for knob in AT.KNOBS:
        for v in AT.candidates(knob, 148):
            c = dataclasses.replace(AT.Choice(), **{knob: v})
            t = BB.BatchTuning(**c.as_dict())
            assert getattr(t, knob) == v
