// bsam_host.cpp -- host driver above the C ABI.
//
// The reference's host side is the Fortran driver: BSAMSolver builds the root
// grid and the below-root multigrid levels (RootInit, CreateBelowSeedLevels,
// InitSeed: lib/bsamroutines.f90:51-176, 205-494; lib/treeops.f90:193-289)
// and TakeTimeSteps calls MultigridIterations once per step
// (lib/bsamroutines.f90:582-789).  No Fortran compiler exists in this image,
// so this file restates that driver in C++ for uniform root grids
// (maxlevel = 0) and calls the C ABI exactly where the Fortran would.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <string>
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


// Fortran edit descriptors of the frame file, as gfortran writes them.
// Fw.d: fixed, right-justified in w columns, a leading "0." kept.
void put_f(std::string& o, double x, int w, int d) {
  char b[64];
  std::snprintf(b, sizeof b, "%*.*f", w, d, x);
  o += b;
}
// ESw.d: one nonzero digit before the point, d after, a two-digit exponent
// written "E+nn"; a three-digit exponent drops the E ("+nnn").
void put_es(std::string& o, double x, int w, int d) {
  char b[64];
  std::snprintf(b, sizeof b, "%.*E", d, x);
  std::string t(b);
  const size_t e = t.find('E');
  if (e != std::string::npos && t.size() - e - 2 > 2) t.erase(e, 1);
  if ((int)t.size() < w) t.insert(0, (size_t)(w - (int)t.size()), ' ');
  o += t;
}
void put_i(std::string& o, int v, int w) {
  char b[32];
  std::snprintf(b, sizeof b, "%*d", w, v);
  o += b;
}

// OutputQ of one patch (lib/bsaminputoutput.f90:78-131) with WriteQ2D/3D
// (133-172): q is the patch's (0:mx+1)^d x nrvars array, column-major.
void output_q(std::string& o, int nd, const bsam_patch_desc& d, const double* xupper,
              const double* q) {
  o += "  \n";  // write(54,*) ' ': a list-directed record, a blank then ' '
  put_i(o, d.level, 3);
  o += ' ';
  put_i(o, nd, 3);
  o += ' ';
  put_i(o, 2, 3);
  o += ' ';
  put_i(o, 2, 3);
  o += '\n';
  const double dx[3] = {d.dx, d.dx, d.dx};
  const double* rows[3] = {dx, d.xlower, xupper};
  for (const double* r : rows) {
    for (int n = 0; n < nd; ++n) {
      if (n) o += ' ';
      put_f(o, r[n], 25, 12);
    }
    o += '\n';
  }
  for (int n = 0; n < nd; ++n) {
    if (n) o += ' ';
    put_i(o, d.mx[n], 8);
  }
  o += '\n';
  for (int n = 0; n < nd; ++n)
    for (int s = 0; s < 2; ++s) {
      if (n || s) o += ' ';
      put_i(o, d.mglobal[n][s], 8);
    }
  o += '\n';
  const int e0 = d.mx[0] + 2, e1 = d.mx[1] + 2, e2 = nd == 3 ? d.mx[2] + 2 : 1;
  const size_t plane = (size_t)e0 * e1 * e2;
  // 10(es20.12,2x) in 2D, 10(f25.12,2x) in 3D; the 2x after the last value
  // is a pending skip that ends with the record.
  for (size_t c = 0; c < plane; ++c) {
    for (int v = 0; v < 2; ++v) {
      if (v) o += "  ";
      if (nd == 2) put_es(o, q[c + v * plane], 20, 12);
      else put_f(o, q[c + v * plane], 25, 12);
    }
    o += '\n';
  }
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

extern "C++" {
namespace {

using Box6 = std::array<int, 6>;  // lo, hi per dimension

// NewSubGrids (lib/bsamroutines.f90:1352-1579) over a patch of extent m,
// with count(box) the number of flagged cells in a box (GridFlagRatio's
// numerator; GetSignatures' entries are the counts of one-cell slabs).
template <class Count>
int new_subgrids_impl(int nd, const int* m, Count count, double desfill, int mgp, int* boxes,
                      int maxboxes) {
  using Box = Box6;
  auto fill_ratio = [&](const Box& b) {
    long cells = 1;
    for (int n = 0; n < nd; ++n) cells *= b[2 * n + 1] - b[2 * n] + 1;
    return (double)count(b) / (double)cells;
  };
  const int maxm = std::max(m[0], std::max(m[1], nd == 3 ? m[2] : 1));
  std::vector<long> sig(3 * (size_t)(maxm + 2), 0), dd(3 * (size_t)(maxm + 2), 0);
  auto SIG = [&](int n, int i) -> long& { return sig[(size_t)n * (maxm + 2) + i]; };
  auto DD = [&](int n, int i) -> long& { return dd[(size_t)n * (maxm + 2) + i]; };
  auto signatures = [&](const Box& b) {  // GetSignatures
    for (int n = 0; n < nd; ++n)
      for (int i = b[2 * n]; i <= b[2 * n + 1]; ++i) {
        Box slab = b;
        slab[2 * n] = slab[2 * n + 1] = i;
        SIG(n, i) = count(slab);
      }
  };
  Box whole = {1, m[0], 1, m[1], 1, m[2]};
  if (fill_ratio(whole) < 1.0e-10) return 0;
  constexpr int kMaxGrids = 1024, kMaxPasses = 15;  // maxsubgrids, maxsplitpasses
  std::vector<Box> grids{whole};
  std::vector<bool> splittable{true};
  for (size_t g = 0; (int)grids.size() < kMaxGrids && g < grids.size(); ++g) {
    for (int pass = 0; splittable[g] && pass < kMaxPasses; ++pass) {
      Box b = grids[g];
      signatures(b);
      for (int n = 0; n < nd; ++n) {  // trim empty ends, down to mgp cells
        int lo = b[2 * n], hi = b[2 * n + 1];
        while (SIG(n, lo) == 0 && lo < b[2 * n + 1] && hi - lo + 1 > mgp) ++lo;
        while (SIG(n, hi) == 0 && hi > b[2 * n] && hi - lo + 1 > mgp) --hi;
        b[2 * n] = lo;
        b[2 * n + 1] = hi;
      }
      grids[g] = b;
      if (fill_ratio(b) >= desfill) {
        splittable[g] = false;
        continue;
      }
      signatures(b);
      int cut_dim = -1, cut = 0;
      for (int n = 0; n < nd && cut_dim < 0; ++n) {  // a hole
        const int lo = b[2 * n], hi = b[2 * n + 1];
        for (int i = lo + mgp; i <= hi - mgp; ++i)
          if (SIG(n, i) == 0 && std::min(i - lo + 1, hi - i) >= mgp) {
            cut_dim = n;
            cut = i;
            break;
          }
      }
      if (cut_dim < 0) {  // the strongest inflection; ties go to the most central
        for (int n = 0; n < nd; ++n)
          for (int i = b[2 * n] + 1; i <= b[2 * n + 1] - 1; ++i)
            DD(n, i) = SIG(n, i - 1) - 2 * SIG(n, i) + SIG(n, i + 1);
        long best = 0;
        int best_dist = 0;
        for (int n = 0; n < nd; ++n) {
          const int lo = b[2 * n], hi = b[2 * n + 1];
          for (int i = lo + std::max(2, mgp); i <= hi - std::max(1, mgp - 1); ++i) {
            const long jump = std::labs(DD(n, i) - DD(n, i - 1));
            const int dist = std::min(i - lo, hi - i + 1);
            if (jump > best || (jump == best && best > 0 && dist > best_dist)) {
              best = jump;
              cut_dim = n;
              cut = i - 1;
              best_dist = dist;
            }
          }
        }
      }
      if (cut_dim < 0) {
        splittable[g] = false;
        continue;
      }
      const int lo = b[2 * cut_dim], hi = b[2 * cut_dim + 1];
      if (std::min(hi - cut, cut - lo + 1) >= mgp) {
        Box upper = b;
        upper[2 * cut_dim] = cut + 1;
        grids[g][2 * cut_dim + 1] = cut;
        grids.push_back(upper);
        splittable.push_back(true);
      }
    }
  }
  if ((int)grids.size() > maxboxes) return BSAM_ERR_ARG;
  for (size_t g = 0; g < grids.size(); ++g)
    for (int e = 0; e < 6; ++e) boxes[6 * g + e] = e / 2 < nd ? grids[g][e] : 1;
  return (int)grids.size();
}
}  // namespace
}  // extern "C++"

int bsam_host_new_subgrids(int ndims, const int* mx, const uint8_t* flags, double desfill,
                           int mgp, int* boxes, int maxboxes) {
  if ((ndims != 2 && ndims != 3) || !mx || !flags || !boxes || maxboxes < 0 || mgp < 1)
    return BSAM_ERR_ARG;
  const int nd = ndims;
  const int m[3] = {mx[0], mx[1], nd == 3 ? mx[2] : 1};
  for (int n = 0; n < 3; ++n)
    if (m[n] < 1) return BSAM_ERR_ARG;
  // Flagged cells in a box, by visiting them.
  auto count = [&](const Box6& b) {
    long s = 0;
    for (int k = b[4]; k <= b[5]; ++k)
      for (int j = b[2]; j <= b[3]; ++j) {
        const uint8_t* row = flags + (size_t)m[0] * ((j - 1) + (size_t)m[1] * (k - 1));
        for (int i = b[0]; i <= b[1]; ++i) s += row[i - 1] != 0;
      }
    return s;
  };
  return new_subgrids_impl(nd, m, count, desfill, mgp, boxes, maxboxes);
}

int bsam_host_new_subgrids_sat(int ndims, const int* mx, const int32_t* sat, double desfill,
                               int mgp, int* boxes, int maxboxes) {
  if ((ndims != 2 && ndims != 3) || !mx || !sat || !boxes || maxboxes < 0 || mgp < 1)
    return BSAM_ERR_ARG;
  const int nd = ndims;
  const int m[3] = {mx[0], mx[1], nd == 3 ? mx[2] : 1};
  for (int n = 0; n < 3; ++n)
    if (m[n] < 1) return BSAM_ERR_ARG;
  // S(i, j, k) = flagged cells in (1:i, 1:j, 1:k), 0 when an index is 0.
  auto S = [&](int i, int j, int k) -> long {
    if (i <= 0 || j <= 0 || k <= 0) return 0;
    return sat[(i - 1) + (size_t)m[0] * ((j - 1) + (size_t)m[1] * (k - 1))];
  };
  // Flagged cells in a box, by inclusion-exclusion over its corners.
  auto count = [&](const Box6& b) {
    const int i0 = b[0] - 1, i1 = b[1], j0 = b[2] - 1, j1 = b[3], k0 = b[4] - 1, k1 = b[5];
    long c = S(i1, j1, k1) - S(i0, j1, k1) - S(i1, j0, k1) + S(i0, j0, k1);
    if (nd == 3) c -= S(i1, j1, k0) - S(i0, j1, k0) - S(i1, j0, k0) + S(i0, j0, k0);
    return c;
  };
  return new_subgrids_impl(nd, m, count, desfill, mgp, boxes, maxboxes);
}

int bsam_host_buffer_flags(int ndims, int npatch, const int* mx, const int* mglobal,
                           uint8_t* flags, int ibuffer) {
  if ((ndims != 2 && ndims != 3) || npatch < 0 || (npatch > 0 && (!mx || !mglobal || !flags)) ||
      ibuffer < 0)
    return BSAM_ERR_ARG;
  if (ibuffer == 0 || npatch == 0) return BSAM_OK;
  const int nd = ndims;
  std::vector<size_t> off(npatch + 1, 0);
  for (int p = 0; p < npatch; ++p) {
    size_t cells = 1;
    for (int n = 0; n < nd; ++n) {
      if (mx[3 * p + n] < 1) return BSAM_ERR_ARG;
      cells *= (size_t)mx[3 * p + n];
    }
    off[p + 1] = off[p] + cells;
  }
  // BufferAndList: a cell flagged on entry whose buffer box lies inside its
  // patch flags that box there; one whose box crosses the patch's edge is
  // listed by global index.  The result is the union of the boxes of every
  // flagged cell, clipped to each patch.
  const std::vector<uint8_t> orig(flags, flags + off[npatch]);
  std::vector<std::array<int, 3>> listed;
  for (int p = 0; p < npatch; ++p) {
    const int m0 = mx[3 * p], m1 = mx[3 * p + 1], m2 = nd == 3 ? mx[3 * p + 2] : 1;
    for (int k = 0; k < m2; ++k)
      for (int j = 0; j < m1; ++j)
        for (int i = 0; i < m0; ++i) {
          if (!orig[off[p] + i + (size_t)m0 * (j + (size_t)m1 * k)]) continue;
          const bool inside = i - ibuffer >= 0 && i + ibuffer < m0 && j - ibuffer >= 0 &&
                              j + ibuffer < m1 &&
                              (nd == 2 || (k - ibuffer >= 0 && k + ibuffer < m2));
          if (!inside) {
            listed.push_back({mglobal[6 * p] + i, mglobal[6 * p + 2] + j,
                              nd == 3 ? mglobal[6 * p + 4] + k : 1});
            continue;
          }
          const int kb = nd == 3 ? ibuffer : 0;
          for (int kk = k - kb; kk <= k + kb; ++kk)
            for (int jj = j - ibuffer; jj <= j + ibuffer; ++jj)
              for (int ii = i - ibuffer; ii <= i + ibuffer; ++ii)
                flags[off[p] + ii + (size_t)m0 * (jj + (size_t)m1 * kk)] = 1;
        }
  }
  // InflateEdgeTags / BufferTaggedCells: each listed cell's box, clipped, on
  // every patch of the level.
  for (const auto& c : listed)
    for (int p = 0; p < npatch; ++p) {
      int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
      bool hit = true;
      for (int n = 0; n < nd; ++n) {
        lo[n] = std::max(c[n] - ibuffer, mglobal[6 * p + 2 * n]);
        hi[n] = std::min(c[n] + ibuffer, mglobal[6 * p + 2 * n + 1]);
        hit = hit && lo[n] <= hi[n];
      }
      if (!hit) continue;
      const int m0 = mx[3 * p], m1 = mx[3 * p + 1];
      const int k0 = nd == 3 ? lo[2] - mglobal[6 * p + 4] : 0;
      const int k1 = nd == 3 ? hi[2] - mglobal[6 * p + 4] : 0;
      for (int k = k0; k <= k1; ++k)
        for (int j = lo[1] - mglobal[6 * p + 2]; j <= hi[1] - mglobal[6 * p + 2]; ++j)
          for (int i = lo[0] - mglobal[6 * p]; i <= hi[0] - mglobal[6 * p]; ++i)
            flags[off[p] + i + (size_t)m0 * (j + (size_t)m1 * k)] = 1;
    }
  return BSAM_OK;
}

int bsam_host_child_desc(int ndims, const bsam_patch_desc* parent, int parent_index,
                         const int* box, bsam_patch_desc* child) {
  if ((ndims != 2 && ndims != 3) || !parent || !box || !child) return BSAM_ERR_ARG;
  bsam_patch_desc c{};
  c.level = parent->level + 1;
  c.parent = parent_index;
  c.dx = parent->dx / 2.0;
  for (int n = 0; n < 3; ++n) {
    c.mx[n] = 1;
    c.mbounds[n][0] = c.mbounds[n][1] = 1;
    c.mglobal[n][0] = c.mglobal[n][1] = 1;
    c.xlower[n] = 0.0;
  }
  for (int f = 0; f < 6; ++f) c.mthbc[f] = 999;  // internalbc
  for (int n = 0; n < ndims; ++n) {
    const int lo = box[2 * n], hi = box[2 * n + 1];
    if (lo < 1 || hi < lo || hi > parent->mx[n]) return BSAM_ERR_ARG;
    c.mx[n] = (hi - lo + 1) * 2;
    c.mbounds[n][0] = lo;
    c.mbounds[n][1] = hi;
    const int glo = parent->mglobal[n][0] + lo - 1, ghi = glo + hi - lo;
    c.mglobal[n][0] = (glo - 1) * 2 + 1;
    c.mglobal[n][1] = ghi * 2;
    if (parent->mthbc[2 * n] < 999 && lo == 1) c.mthbc[2 * n] = parent->mthbc[2 * n];
    if (parent->mthbc[2 * n + 1] < 999 && hi == parent->mx[n])
      c.mthbc[2 * n + 1] = parent->mthbc[2 * n + 1];
    c.xlower[n] = (double)(lo - 1) * parent->dx + parent->xlower[n];
  }
  *child = c;
  return BSAM_OK;
}


int bsam_host_format_frame(const char* path, int ndims, double time, int finestlevel,
                           int npatch, const bsam_patch_desc* patches, const double* const* q) {
  if (!path || (ndims != 2 && ndims != 3) || npatch < 0 || (npatch > 0 && (!patches || !q)))
    return BSAM_ERR_ARG;
  std::string o;
  put_f(o, time, 25, 12);
  o += '\n';
  put_i(o, finestlevel, 3);
  o += '\n';
  // Levels rootlevel .. finestlevel, table (ApplyOnLevel) order within each.
  for (int level = 0; level <= finestlevel; ++level)
    for (int p = 0; p < npatch; ++p) {
      const bsam_patch_desc& d = patches[p];
      if (d.level != level) continue;
      if (!q[p]) return BSAM_ERR_ARG;
      // xupper: the root's is xlower + mx dx; a refined patch's is
      // mbounds(:,2) * parent dx + parent xlower (MakeNewGrid).
      double xu[3] = {0.0, 0.0, 0.0};
      for (int n = 0; n < ndims; ++n) {
        if (d.level == 0 || d.parent < 0 || d.parent >= npatch) {
          xu[n] = d.xlower[n] + d.mx[n] * d.dx;
        } else {
          const bsam_patch_desc& pd = patches[d.parent];
          xu[n] = (double)d.mbounds[n][1] * pd.dx + pd.xlower[n];
        }
      }
      output_q(o, ndims, d, xu, q[p]);
    }
  FILE* f = std::fopen(path, "wb");
  if (!f) return BSAM_ERR_ARG;
  const size_t w = std::fwrite(o.data(), 1, o.size(), f);
  const int rc = std::fclose(f);
  return (w == o.size() && rc == 0) ? BSAM_OK : BSAM_ERR_ARG;
}

int bsam_host_write_frame(bsam_gpu* h, const char* path, int ndims, double time, int npatch,
                          const bsam_patch_desc* patches) {
  if (!h || !path || (ndims != 2 && ndims != 3) || npatch <= 0 || !patches) return BSAM_ERR_ARG;
  const int nd = ndims;
  int finest = 0;
  for (int p = 0; p < npatch; ++p) finest = std::max(finest, patches[p].level);
  std::vector<std::vector<double>> store(npatch);
  std::vector<const double*> q(npatch, nullptr);
  for (int p = 0; p < npatch; ++p) {
    const bsam_patch_desc& d = patches[p];
    if (d.level < 0) continue;
    size_t n = 2;
    for (int k = 0; k < nd; ++k) n *= (size_t)(d.mx[k] + 2);
    store[p].resize(n);
    const int rc = bsam_gpu_get_field(h, p, BSAM_FIELD_Q, store[p].data());
    if (rc != BSAM_OK) return rc;
    q[p] = store[p].data();
  }
  return bsam_host_format_frame(path, nd, time, finest, npatch, patches, q.data());
}


struct bsam_amr {
  bsam_gpu* h = nullptr;
  int nd = 2;
  bsam_regrid_params p{};
  std::vector<bsam_patch_desc> table;
  bool firstamr = true;
  std::vector<int32_t> sat;  // summed-area tables of a level's buffered flags
  std::vector<int> boxes;
  // Host wall-clock seconds per phase, summed over steps (bsam_amr_profile).
  double t[BSAM_AMR_NPHASE] = {0};
  int64_t steps = 0;
};

namespace {
struct PhaseClock {
  double* acc;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  explicit PhaseClock(double* a) : acc(a) {}
  void lap(int phase) {
    const auto t1 = std::chrono::steady_clock::now();
    acc[phase] += std::chrono::duration<double>(t1 - t0).count();
    t0 = t1;
  }
};
}  // namespace

int bsam_amr_create(bsam_amr** out, bsam_gpu* h, int ndims, const bsam_regrid_params* p,
                    int npatch, const bsam_patch_desc* patches) {
  if (!out || !h || !p || (ndims != 2 && ndims != 3) || npatch <= 0 || !patches ||
      p->maxlevel < 0 || p->maxlevel > BSAM_AMR_MAXLEVEL)
    return BSAM_ERR_ARG;
  for (int l = 0; l < p->maxlevel; ++l)
    if (p->ibuffer[l] < 0 || p->minimumgridpoints[l] < 1 || !(p->desiredfillratios[l] > 0.0))
      return BSAM_ERR_ARG;
  auto* a = new bsam_amr();
  a->h = h;
  a->nd = ndims;
  a->p = *p;
  a->table.assign(patches, patches + npatch);
  int finest = 0;
  for (const auto& d : a->table) finest = std::max(finest, d.level);
  // BSAMSolver: SetGhost on every level, CopyQToQold (bsamroutines.f90:144-147).
  for (int level = 0; level <= finest; ++level) {
    const int rc = bsam_gpu_set_ghost_level(h, level);
    if (rc) {
      delete a;
      return rc;
    }
  }
  const int rc = bsam_gpu_copy_q_to_qold(h);
  if (rc) {
    delete a;
    return rc;
  }
  *out = a;
  return BSAM_OK;
}

}  // extern "C"

namespace {

// AMR(rootlevel) and what TakeTimeSteps does before MultigridIterations
// (lib/bsamroutines.f90:646-661): the first half of a time step.
int amr_regrid_part(bsam_amr* a, PhaseClock& clk) {
  bsam_gpu* h = a->h;
  const int nd = a->nd;
  const std::vector<bsam_patch_desc> start = a->table;
  std::vector<bsam_patch_desc> table = a->table;
  // The old grids of the refined levels as TransferValues reads them.
  int rc = bsam_gpu_stash(h);
  if (rc) return rc;
  clk.lap(BSAM_AMR_PHASE_STASH);
  rc = bsam_gpu_set_ghost_level(h, 0);  // AMR(rootlevel)
  if (rc) return rc;
  clk.lap(BSAM_AMR_PHASE_GHOST);
  // EstimateLevelErrors(0)'s restriction of the root into the level below and
  // that level's SetGhost are not issued: the V-cycle restricts the root again
  // before it reads that level, and qold below the root is never read.
  for (int L = 0; L < a->p.maxlevel; ++L) {
    if (L >= 1) {
      rc = bsam_gpu_restrict_level(h, L);  // EstimateLevelErrors(L)
      if (rc) return rc;
      clk.lap(BSAM_AMR_PHASE_GHOST);
    }
    std::vector<int> lvl;
    size_t cells = 0;
    for (int i = 0; i < (int)table.size(); ++i)
      if (table[i].level == L) {
        lvl.push_back(i);
        size_t c = 1;
        for (int n = 0; n < nd; ++n) c *= (size_t)table[i].mx[n];
        cells += c;
      }
    // Tagging, BufferAndList + InflateEdgeTags and the summed-area tables
    // NewSubGrids counts from, all of the level on the device.
    a->sat.assign(cells, 0);
    rc = bsam_gpu_tag_level(h, L, a->p.qtolerance[L], a->p.ibuffer[L], a->sat.data());
    if (rc) return rc;
    std::vector<int> mx(3 * lvl.size());
    for (size_t k = 0; k < lvl.size(); ++k)
      for (int n = 0; n < 3; ++n) mx[3 * k + n] = table[lvl[k]].mx[n];
    clk.lap(BSAM_AMR_PHASE_TAG);
    // GridAdapt(L): RefineGrid -> NewSubGrids per patch, MakeNewGrid per box.
    std::vector<bsam_patch_desc> made;
    size_t off = 0;
    for (size_t k = 0; k < lvl.size(); ++k) {
      const bsam_patch_desc& par = table[lvl[k]];
      size_t c = 1;
      for (int n = 0; n < nd; ++n) c *= (size_t)par.mx[n];
      // The boxes are disjoint and each holds a flagged cell: at most c.
      const int cap = (int)c;
      if (a->boxes.size() < 6 * c) a->boxes.resize(6 * c);
      const int nb = bsam_host_new_subgrids_sat(nd, &mx[3 * k], a->sat.data() + off,
                                                a->p.desiredfillratios[L],
                                                a->p.minimumgridpoints[L], a->boxes.data(), cap);
      if (nb < 0) return nb;
      for (int b = 0; b < nb; ++b) {
        int box[6];
        for (int n = 0; n < 3; ++n) {
          box[2 * n] = a->boxes[6 * b + 2 * n];
          box[2 * n + 1] = a->boxes[6 * b + 2 * n + 1];
        }
        bsam_patch_desc child;
        rc = bsam_host_child_desc(nd, &par, lvl[k], box, &child);
        if (rc) return rc;
        made.push_back(child);
      }
      off += c;
    }
    // Levels <= L keep their grids; level L + 1 becomes the new grids,
    // youngest first (TreeOps prepends); deeper levels lose their grids.
    std::vector<int> keep, index(table.size(), -1);
    for (int i = 0; i < (int)table.size(); ++i)
      if (table[i].level <= L) {
        index[i] = (int)keep.size();
        keep.push_back(i);
      }
    std::vector<bsam_patch_desc> next;
    std::vector<int> carry;
    for (int i : keep) {
      bsam_patch_desc d = table[i];
      d.parent = d.parent >= 0 ? index[d.parent] : -1;
      next.push_back(d);
      carry.push_back(i);
    }
    for (auto it = made.rbegin(); it != made.rend(); ++it) {
      bsam_patch_desc d = *it;
      d.parent = index[d.parent];
      next.push_back(d);
      carry.push_back(-1);
    }
    // TransferValues: each new grid with each old grid of its level.
    std::vector<int> transfers;
    for (int c = (int)keep.size(); c < (int)next.size(); ++c)
      for (int o = 0; o < (int)start.size(); ++o) {
        if (start[o].level != L + 1) continue;
        bool overlap = true;
        for (int n = 0; n < nd; ++n)
          overlap = overlap && std::max(next[c].mglobal[n][0], start[o].mglobal[n][0]) <=
                                   std::min(next[c].mglobal[n][1], start[o].mglobal[n][1]);
        if (overlap) {
          transfers.push_back(c);
          transfers.push_back(o);
        }
      }
    int finest = 0;
    for (const auto& d : next) finest = std::max(finest, d.level);
    clk.lap(BSAM_AMR_PHASE_CLUSTER);
    rc = bsam_gpu_regrid(h, (int)next.size(), next.data(), finest, carry.data(),
                         (int)transfers.size() / 2, transfers.data());
    if (rc) return rc;
    clk.lap(BSAM_AMR_PHASE_REGRID);
    table.swap(next);
    a->table = table;
    if (made.empty()) {
      // AMR(L + 1) on an empty level: EstimateLevelErrors(L + 1) still sets
      // the ghosts of level L.
      if (L + 1 < a->p.maxlevel) {
        rc = bsam_gpu_set_ghost_level(h, L);
        if (rc) return rc;
      }
      clk.lap(BSAM_AMR_PHASE_GHOST);
      break;
    }
    rc = bsam_gpu_set_ghost_level(h, L + 1);  // AMR(L + 1)
    if (rc) return rc;
    clk.lap(BSAM_AMR_PHASE_GHOST);
  }
  a->table = table;
  if (a->firstamr) {
    rc = bsam_gpu_fill_down(h);
    if (rc) return rc;
    a->firstamr = false;
  }
  return bsam_gpu_copy_q_to_qold(h);
}

}  // namespace

namespace bsam {
// The engine a native AMR driver steps (declared in engine_view.h, which
// holds device code and is not included by host-compiled sources).
bsam_gpu* amr_engine(bsam_amr* a);
bsam_gpu* amr_engine(bsam_amr* a) { return a ? a->h : nullptr; }
}  // namespace bsam

extern "C" {

int bsam_amr_regrid(bsam_amr* a) {
  if (!a) return BSAM_ERR_ARG;
  PhaseClock clk(a->t);
  return amr_regrid_part(a, clk);
}

int bsam_amr_step(bsam_amr* a, int* nvcycles, double* residual, int* converged) {
  if (!a) return BSAM_ERR_ARG;
  bsam_gpu* h = a->h;
  PhaseClock clk(a->t);
  int rc = amr_regrid_part(a, clk);
  if (rc) return rc;
  int nv = 0, conv = 0;
  double res = 0.0;
  rc = bsam_gpu_multigrid_iterations(h, &nv, &res, &conv);
  clk.lap(BSAM_AMR_PHASE_SOLVE);
  ++a->steps;
  if (nvcycles) *nvcycles = nv;
  if (residual) *residual = res;
  if (converged) *converged = conv;
  return rc;
}

int bsam_amr_profile(const bsam_amr* a, double* seconds, int n) {
  if (!a || !seconds || n < 0) return BSAM_ERR_ARG;
  for (int i = 0; i < n && i < BSAM_AMR_NPHASE; ++i) seconds[i] = a->t[i];
  return (int)a->steps;
}

int bsam_amr_table(const bsam_amr* a, bsam_patch_desc* out, int maxn) {
  if (!a) return BSAM_ERR_ARG;
  const int n = (int)a->table.size();
  if (out)
    for (int i = 0; i < n && i < maxn; ++i) out[i] = a->table[i];
  return n;
}

void bsam_amr_destroy(bsam_amr* a) { delete a; }

}  // extern "C"
