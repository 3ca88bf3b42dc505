// problem.cuh -- the problem module the kernels are compiled for.
//
// The reference links one user problem module (problems/<name>/problem.f90)
// into the multigrid library; the library calls its routines by fixed names.
// Here a problem module is a trait type whose static members are those
// routines' device twins, and `Problem` names the one this build uses.  The
// default is CahnHilliard (problem_ch.cuh); another module is chosen at
// compile time with
//
//   -DBSAM_PROBLEM_HEADER='"my_problem.cuh"' -DBSAM_PROBLEM=MyProblem
//
// A module provides (T = float or double, D = 2 or 3):
//   nrvars, maux, errortype     sizes of the reference's problem data
//   paired_f32                  whether relax_pair_f32 (fused2.cuh) may pair
//                               its FP32 Newton step; false gives the fused
//                               stage the scalar RelaxCell per cell
//   Stencil<T, D>               a cell's neighbourhood (phi, mu)
//   RelaxCell<T, D, DELTA>      RelaxGrid2D/3D at one cell (DELTA: the
//                               correction form of the mixed precision)
//   OperatorCell<T, D, DELTA>   Operator2D/3D at one cell
//   SourceCell<T>               Source2D/3D + UpdateSourceFunction
//   Dfc, D2fc, Dfe, Ff          the free-energy terms (energy statistics)
//   TagCell<D>                  SetErrFlagsUser2D/3D's test
#pragma once

#ifdef BSAM_PROBLEM_HEADER
#include BSAM_PROBLEM_HEADER
#else
#include "problem_ch.cuh"
#endif

#ifndef BSAM_PROBLEM
#define BSAM_PROBLEM CahnHilliard
#endif

namespace bsam {

using Problem = BSAM_PROBLEM;

// The engine stores two components per cell (q(:,:,1:2)) and no auxiliary
// fields, and tags with the user routine.
static_assert(Problem::nrvars == 2, "the device layout holds two components per cell");
static_assert(Problem::maux == 0, "no auxiliary fields on the device");
static_assert(Problem::errortype == 1, "tagging by the problem's own test");

}  // namespace bsam
