"""The problem module is a compile-time trait: the kernels compile against a
module other than the default (here one that forbids the paired FP32 update,
so the fused stage takes the module's scalar RelaxCell), and the selection
and the scalar fallback are the ones the build picked (compile-time
asserts).  Compile only: no GPU needed."""
import os
import shutil
import subprocess

import pytest

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "bsam_b200",
                    "csrc")

ALT = """#pragma once
#include "problem_ch.cuh"
namespace bsam {
// A second module: Cahn-Hilliard's routines without the paired FP32 update.
struct AltProblem : CahnHilliard {
  static constexpr bool paired_f32 = false;
};
}  // namespace bsam
"""

TU = """#include "batch.cuh"
#include "defect2.cuh"
#include "fused2.cuh"
#include "regrid.cuh"
#include "stats.cuh"
namespace bsam {
static_assert(std::is_same<Problem, %(prob)s>::value, "the module the build chose");
static_assert(std::is_same<RelaxPair<float, true>, %(pair)s>::value, "the pair form");
template __global__ void kb_smooth2<float, true, 4, 1>(const DevPatch*, const Item*, const int*,
                                                       int, int, int, int, int, int*, TileRuns);
template __global__ void kb_smooth2<double, false, 4, 1>(const DevPatch*, const Item*,
                                                         const int*, int, int, int, int, int,
                                                         int*, TileRuns);
template __global__ void kb_defect_tma<2>(const DevPatch*, const Item*, const int*, double*, int,
                                          int*, TileRuns);
template __global__ void k_errflags_list<3>(const DevPatch*, const FlagTask*, double, uint8_t*);
template __global__ void k_stats<2>(const DevPatch*, const StatBlock*, double*);
}  // namespace bsam
"""


def nvcc():
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    return None


def compile_tu(tmp_path, prob, pair, defines):
    (tmp_path / "alt_problem.cuh").write_text(ALT)
    (tmp_path / "tu.cu").write_text(TU % {"prob": prob, "pair": pair})
    cmd = [nvcc(), "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "--fmad=false",
           f"-I{CSRC}", f"-I{tmp_path}", *defines, "-c", str(tmp_path / "tu.cu"), "-o",
           str(tmp_path / "tu.o")]
    return subprocess.run(cmd, capture_output=True, text=True)


@pytest.mark.skipif(nvcc() is None, reason="nvcc not found")
def test_kernels_compile_against_another_module(tmp_path):
    r = compile_tu(tmp_path, "AltProblem", "RelaxPairScalar<float, true>",
                   ['-DBSAM_PROBLEM_HEADER="alt_problem.cuh"', "-DBSAM_PROBLEM=AltProblem"])
    assert r.returncode == 0, r.stderr[-2000:]


@pytest.mark.skipif(nvcc() is None, reason="nvcc not found")
def test_default_module_is_cahn_hilliard_with_paired_update(tmp_path):
    r = compile_tu(tmp_path, "CahnHilliard", "RelaxPairF32<true>", [])
    assert r.returncode == 0, r.stderr[-2000:]
