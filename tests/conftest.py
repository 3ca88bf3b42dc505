import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    import pyoracle
    pyoracle.build()
    return pyoracle


def _has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_lib():
    """The native library, built in-tree; GPU tests fail (not skip) without it."""
    import bsam_b200
    from bsam_b200 import build as B
    B.build()
    if not _has_cuda():
        pytest.fail("gpu test selected but no CUDA device is visible")
    return bsam_b200.lib()


GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_hierarchy(name):
    """The hierarchy of a tests/golden/ref_mg_*.npz fixture (patch records,
    initial q of every patch on a level >= 0) and the fixture itself."""
    import numpy as np
    from bsam_b200 import amr
    d = np.load(os.path.join(GOLD, f"ref_{name}.npz"))
    nd = int(d["ndims"])
    descs, q0s, off = [], [], 0
    for i in range(len(d["level"])):
        desc = {"level": int(d["level"][i]), "parent": int(d["parent"][i]),
                "mx": [int(v) for v in d["mx"][i]],
                "mbounds": [[int(v) for v in b] for b in d["mbounds"][i]],
                "mglobal": [[int(v) for v in b] for b in d["mglobal"][i]],
                "mthbc": [int(v) for v in d["mthbc"][i]], "dx": float(d["dxs"][i]),
                "xlower": [float(v) for v in d["xlower"][i]]}
        descs.append(desc)
        if desc["level"] >= 0:
            shape = tuple(m + 2 for m in desc["mx"][:nd]) + (2,)
            n = int(np.prod(shape))
            q0s.append(d["q0"][off:off + n].reshape(shape, order="F"))
            off += n
    hier = amr.Hierarchy(ndims=nd, descs=descs, q0s=q0s, dt=float(d["hdt"]),
                         eps=float(d["heps"]), qerrortol=float(d["qerrortol"]),
                         maxvcycles=int(d["maxvcycles"]),
                         nsmoothingpasses=int(d["nsmoothingpasses"]))
    return hier, d


@pytest.fixture(scope="session")
def golden_hier():
    return golden_hierarchy


@pytest.fixture(scope="session")
def gpu_free_lib():
    """The native library for host-only entry points (no device needed)."""
    import bsam_b200
    from bsam_b200 import build as B
    B.build()
    return bsam_b200.lib()
