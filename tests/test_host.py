"""Host driver (C++ restatement of RootInit / InitSeed) without a GPU."""
import numpy as np
import pytest

import bsam_b200 as B
from bsam_b200 import workloads as W


@pytest.fixture(scope="module", autouse=True)
def _built():
    from bsam_b200 import build
    build.build()


def test_uniform_hierarchy_matches_initseed():
    prob = W.config1(nsteps=1, n=128)
    arr, n = B.build_uniform(prob)
    assert n == 8                      # 128 -> 1: minlevel = -7
    levels = [arr[i].level for i in range(n)]
    assert levels == [0, -1, -2, -3, -4, -5, -6, -7]
    for i in range(n):
        d = arr[i]
        assert d.mx[0] == 128 >> i and d.mx[1] == 128 >> i and d.mx[2] == 1
        assert d.dx == pytest.approx(1.0 / 128 * 2 ** i, rel=0, abs=0)
        assert d.parent == (i + 1 if i + 1 < n else -1)
        if d.parent >= 0:
            assert tuple(d.mbounds[0]) == (1, d.mx[0] // 2)


def test_odd_coarsest_and_3d():
    arr, n = B.build_uniform(W.config1(nsteps=1, n=96))
    assert n == 6 and arr[n - 1].mx[0] == 3
    p3 = W.config3(nsteps=1, n=32)
    arr, n = B.build_uniform(p3)
    assert n == 6 and arr[0].mx[2] == 32 and arr[5].mx[2] == 1


def test_rejects_odd_root():
    prob = W.config1(nsteps=1, n=128)
    prob.mx = (127, 128, 1)
    with pytest.raises(B.BsamError):
        B.build_uniform(prob)
