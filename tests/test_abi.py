"""The C-ABI library loads and exports every symbol include/*.h declares
(no compute call: these run without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for hdr in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(hdr).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(bsam_\w+)\s*\(", text):
            names.add(m.group(1))
    return names


@pytest.fixture(scope="module")
def native():
    from bsam_b200 import build as B
    B.build()
    import bsam_b200
    return bsam_b200.lib()


def test_headers_declare_entry_points():
    names = declared_symbols()
    assert "bsam_gpu_multigrid_iterations" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol(native):
    missing = [n for n in sorted(declared_symbols()) if not hasattr(native, n)]
    assert not missing, missing


def test_python_binding_list_matches_headers():
    import bsam_b200
    assert set(bsam_b200.ABI_SYMBOLS) == declared_symbols()


def test_strerror_needs_no_device(native):
    assert native.bsam_gpu_strerror(0) == b"ok"
    assert native.bsam_gpu_strerror(-5) == b"configuration not supported"


def test_create_rejects_unsupported_without_device(native):
    import bsam_b200 as B
    h = ctypes.c_void_p()
    rp = B.RunParams(ndims=2, nrvars=3, mbc=1, maux=0, nsmoothingpasses=2, maxvcycles=5,
                     errortype=1, precision=0, dt=1e-4, qerrortol=1e-8, alpha=1, eps=0.01)
    assert native.bsam_gpu_create(ctypes.byref(h), 0, ctypes.byref(rp)) == -5
    assert not h.value
