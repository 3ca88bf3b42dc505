"""Build recipe of the native library (sm_100a only).

Compiles bsam_b200/csrc/*.cu into bsam_b200/libbsam_gpu.so with nvcc.  The
FP64 path is built with --fmad=false so that no multiply-add is contracted
and results match the reference arithmetic operation for operation.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libbsam_gpu.so")
SOURCES = ["bsam_gpu.cu", "bsam_host.cpp", "bsam_noalloc.cu", "bsam_batch.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


STAMP = LIB + ".sha256"


def _digest() -> str:
    """Hash of every source and header the library is built from and of this
    recipe: the library is rebuilt when it changes (file times do not survive
    copying the tree to another machine, contents do)."""
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    inc = os.path.join(HERE, "..", "include")
    deps += [os.path.join(inc, f) for f in os.listdir(inc)]
    deps.append(os.path.abspath(__file__))
    h = hashlib.sha256()
    for d in sorted(deps):
        if os.path.isfile(d):
            h.update(os.path.basename(d).encode())
            with open(d, "rb") as f:
                h.update(f.read())
    return h.hexdigest()


def _stale() -> bool:
    if not os.path.exists(LIB) or not os.path.exists(STAMP):
        return True
    with open(STAMP) as f:
        return f.read().strip() != _digest()


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    digest = _digest()
    cmd = [nvcc(), "-O3", "-std=c++17", *ARCH, "-lineinfo", "--fmad=false",
           "-Xcompiler", "-fPIC", "-shared", "-o", LIB,
           *[os.path.join(CSRC, s) for s in SOURCES]]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    with open(STAMP, "w") as f:
        f.write(digest + "\n")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
