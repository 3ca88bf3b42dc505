"""The autotuner on the GPU: a search over a small sample, the cache, and the
results of every searched choice bit-identical to the default's."""
import numpy as np
import pytest

from bsam_b200 import autotune as AT
from bsam_b200 import batch as BB
from bsam_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_search_and_every_choice_bit_identical(gpu_lib, tmp_path):
    probs = [W.seeded(2, n, 0.01, 2, seed=300 + n, cbar=0.5, amp=0.025) for n in (64, 96, 128)]
    path = str(tmp_path / "t.json")
    res = AT.tuned_choice(probs, BB.PREC_MIXED, per_side=1, path=path)
    assert not res["cached"] and res["gain"] >= 1.0
    again = AT.tuned_choice(probs, BB.PREC_MIXED, per_side=1, path=path)
    assert again["cached"] and again["choice"] == res["choice"]
    ref = BB.solve_all(probs, precision=BB.PREC_MIXED)
    for t in res["timings"]:
        got = BB.solve_all(probs, precision=BB.PREC_MIXED, **t["choice"])
        for a, b in zip(ref, got):
            for k in ("q", "nvcycles", "residual"):
                assert np.array_equal(a[k], b[k]), (t["choice"], k)
