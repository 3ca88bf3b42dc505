// bsam_host.cpp -- host driver above the C ABI.
//
// The reference's host side is the Fortran driver: BSAMSolver builds the root
// grid and the below-root multigrid levels (RootInit, CreateBelowSeedLevels,
// InitSeed: lib/bsamroutines.f90:51-176, 205-494; lib/treeops.f90:193-289)
// and TakeTimeSteps calls MultigridIterations once per step
// (lib/bsamroutines.f90:582-789).  No Fortran compiler exists in this image,
// so this file restates that driver in C++ for uniform root grids
// (maxlevel = 0) and calls the C ABI exactly where the Fortran would.
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/bsam_gpu.h"
#include "../../include/bsam_host.h"

namespace {

// minlevel = 1 -> coarsen while every dimension is even, at most 10 times
// (lib/bsamroutines.f90:287-301).
int resolve_minlevel(const bsam_host_grid* g) {
  if (g->minlevel != 1) return g->minlevel;
  int ml = 0, m[3] = {g->mx[0], g->mx[1], g->mx[2]};
  for (;;) {
    bool even = true;
    for (int n = 0; n < g->ndims; ++n) even = even && (m[n] % 2 == 0);
    if (!even || ml == 10) break;
    ++ml;
    for (int n = 0; n < g->ndims; ++n) m[n] /= 2;
  }
  return -ml;
}

}  // namespace

extern "C" {

int bsam_host_levels(const bsam_host_grid* g) {
  if (!g) return BSAM_ERR_ARG;
  return 1 - resolve_minlevel(g);
}

int bsam_host_build_uniform(const bsam_host_grid* g, bsam_patch_desc* out, int maxn,
                            int* npatch) {
  if (!g || !out || !npatch) return BSAM_ERR_ARG;
  const int nd = g->ndims;
  if (nd < 2 || nd > 3) return BSAM_ERR_ARG;
  const int minlevel = resolve_minlevel(g);
  if (minlevel > 0 || minlevel < -10) return BSAM_ERR_ARG;
  const int n = 1 - minlevel;
  if (n > maxn) return BSAM_ERR_ARG;
  double dx[3] = {0, 0, 0};
  for (int d = 0; d < nd; ++d) {
    // RootInit validation (lib/bsamroutines.f90:319-371).
    if (g->mx[d] <= 0 || g->mx[d] % 2 != 0) return BSAM_ERR_ARG;
    if (g->xupper[d] <= g->xlower[d]) return BSAM_ERR_ARG;
    dx[d] = (g->xupper[d] - g->xlower[d]) / (double)g->mx[d];
  }
  for (int d = 1; d < nd; ++d)
    if (std::fabs(dx[0] - dx[d]) > 1.0e-10) return BSAM_ERR_ARG;
  // Patch 0 = root (level 0); patch l = level -l, parent of patch l-1.
  std::memset(out, 0, sizeof(bsam_patch_desc) * n);
  bsam_patch_desc* root = &out[0];
  root->level = 0;
  root->parent = n > 1 ? 1 : -1;
  for (int d = 0; d < 3; ++d) {
    root->mx[d] = d < nd ? g->mx[d] : 1;
    root->mglobal[d][0] = 1;
    root->mglobal[d][1] = root->mx[d];
    root->mbounds[d][0] = 1;
    root->mbounds[d][1] = root->mx[d];
    root->xlower[d] = d < nd ? g->xlower[d] : 0.0;
  }
  for (int f = 0; f < 6; ++f) root->mthbc[f] = g->mthbc[f];
  root->dx = dx[0];
  double h = dx[0];
  for (int l = 1; l < n; ++l) {
    // InitSeed (lib/bsamroutines.f90:426-494): the seed is born from its child.
    bsam_patch_desc* child = &out[l - 1];
    bsam_patch_desc* seed = &out[l];
    seed->level = -l;
    seed->parent = (l + 1 < n) ? l + 1 : -1;
    for (int d = 0; d < 3; ++d) {
      if (d < nd) {
        if (child->mx[d] % 2 != 0) return BSAM_ERR_ARG;
        seed->mx[d] = child->mx[d] / 2;
        seed->mglobal[d][0] = 1;
        seed->mglobal[d][1] = child->mglobal[d][1] / 2;
        child->mbounds[d][0] = 1;
        child->mbounds[d][1] = seed->mx[d];
        seed->mbounds[d][0] = 1;
        seed->mbounds[d][1] = seed->mx[d];
      } else {
        seed->mx[d] = 1;
        seed->mglobal[d][0] = seed->mglobal[d][1] = 1;
        seed->mbounds[d][0] = seed->mbounds[d][1] = 1;
      }
      seed->xlower[d] = child->xlower[d];
    }
    for (int f = 0; f < 6; ++f) seed->mthbc[f] = child->mthbc[f];
    h = h * 2.0;  // seedinfo%dx = child%dx * 2.0
    seed->dx = h;
  }
  *npatch = n;
  return BSAM_OK;
}

int bsam_host_take_time_steps(bsam_gpu* h, int nsteps, int root_patch, double* q_steps,
                              int64_t q_stride, int* nvcycles, double* residuals,
                              int* converged, double* mass) {
  if (!h || nsteps < 0) return BSAM_ERR_ARG;
  for (int step = 0; step < nsteps; ++step) {
    // AMR(rootlevel) on an unchanged hierarchy -> SetGhost(level, 0) from the
    // root up; FillDown(solution) on the first step; CopyQToQold on every
    // level (lib/bsamroutines.f90:648-661).  FillDown repeated at the start
    // of a later call gives the same values (the fine levels are unchanged).
    int rc = bsam_gpu_set_ghost(h);
    if (rc) return rc;
    if (step == 0) {
      rc = bsam_gpu_fill_down(h);
      if (rc) return rc;
    }
    rc = bsam_gpu_copy_q_to_qold(h);
    if (rc) return rc;
    int nv = 0, conv = 0;
    double res = 0.0;
    rc = bsam_gpu_multigrid_iterations(h, &nv, &res, &conv);  // eqfn = 1
    if (nvcycles) nvcycles[step] = nv;
    if (residuals) residuals[step] = res;
    if (converged) converged[step] = conv;
    if (rc) return rc;
    if (q_steps) {
      rc = bsam_gpu_get_field(h, root_patch, BSAM_FIELD_Q, q_steps + step * q_stride);
      if (rc) return rc;
    }
    if (mass) {
      rc = bsam_gpu_mass(h, &mass[step]);
      if (rc) return rc;
    }
  }
  return BSAM_OK;
}

}  // extern "C"
