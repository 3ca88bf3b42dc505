// kernels.cuh -- FAS V-cycle kernels over the device patch table.
//
// One per-cell device function per reference routine on the hot path, and
// two ways of mapping cells to threads:
//  * grid kernels (k_*) take a work list of Items (patch, tile) so that one
//    launch covers every patch of a level.  A CTA is 32 x TILE_Y threads;
//    every thread owns a pair of adjacent cells in x (one red, one black),
//    which keeps warps on 64 contiguous cells of a row;
//  * block loops (bottom.cuh) walk all cells of a small patch with one CTA.
//
// Ghost cells: for patches whose faces are all physical (DevPatch::wt), the
// code that changes a boundary cell also writes the ghost cells SetBC would
// derive from it (write-through).  This reproduces SetGhost's result exactly:
// SetBC2D/3D (boundary.f90:661-885) processes the faces in order and copies
// whole rows including the ghost rows, so a ghost outside in the set S of
// dimensions ends up as the map of each face in S (ascending dimension)
// applied to the interior cell reflected across all of S.
#pragma once
#include "bsam_types.h"
#include "problem.cuh"

namespace bsam {

template <class T> __device__ __forceinline__ T* fld(void* p) { return static_cast<T*>(p); }

// The entries of an n-long work list a CTA takes: runs of `chunk`
// consecutive entries, run r going to CTA r mod gridDim.x (chunk 1 is the
// plain grid-stride order).  A list holds each problem's tiles in a row, so
// the tiles of a run mostly share their patch records, which after the
// run's first tile come from L1 instead of a chain of L2 round trips; the
// order in which a CTA visits tiles changes no result.
struct TileRuns {
  int chunk;
  __device__ __forceinline__ int first() const { return (int)blockIdx.x * chunk; }
  __device__ __forceinline__ int next(int x) const {
    ++x;
    return (x % chunk) != 0 ? x : x + (int)(gridDim.x - 1) * chunk;
  }
};

// The pre-smoothed state of a level: the second buffer when the level's
// stages run the fused kernel (q -> qb -> q), else q itself.
__device__ __forceinline__ void* const* mid_state(const DevPatch& P) {
  return P.fused ? P.qb : P.q;
}

__device__ __forceinline__ int64_t cidx(const DevPatch& P, int i, int j, int k) {
  return (int64_t)i + (int64_t)j * P.sy + (int64_t)k * P.sz;
}

template <class T> __device__ __forceinline__ T bc_map(int code, T v) {
  return code == BC_REFLECT ? T(2) - v : (code == BC_NEGATE ? -v : v);
}

// Choice s of one dimension for a ghost combination: 0 = the cell's own
// coordinate, 1 = the low ghost (fed by coordinate 1 on a physical low face,
// by coordinate n on a periodic one), 2 = the high ghost (fed by coordinate n
// on a physical high face, by coordinate 1 on a periodic one).
__device__ __forceinline__ bool ghost_choice(int s, int co, int n, int lo_code, int hi_code,
                                             int& g, int& code) {
  if (s == 0) {
    g = co;
    code = BC_NONE;
    return true;
  }
  if (s == 1) {
    g = 0;
    code = lo_code;
    if (lo_code == BC_PERIODIC) return co == n;
    return co == 1 && lo_code != BC_NONE;
  }
  g = n + 1;
  code = hi_code;
  if (hi_code == BC_PERIODIC) return co == 1;
  return co == n && hi_code != BC_NONE;
}

// Ghost write-through for the cell (i,j,k) of patch P whose new values are
// (v0, v1).
template <class T, int D>
__device__ __forceinline__ void write_through(const DevPatch& P, T* q0, T* q1, int i, int j,
                                              int k, T v0, T v1) {
#pragma unroll
  for (int sz = 0; sz < (D == 3 ? 3 : 1); ++sz) {
    int gz = k, cz = BC_NONE;
    if (D == 3 && !ghost_choice(sz, k, P.n[2], P.bc[4], P.bc[5], gz, cz)) continue;
#pragma unroll
    for (int sy = 0; sy < 3; ++sy) {
      int gy, cy;
      if (!ghost_choice(sy, j, P.n[1], P.bc[2], P.bc[3], gy, cy)) continue;
#pragma unroll
      for (int sx = 0; sx < 3; ++sx) {
        if (sx == 0 && sy == 0 && sz == 0) continue;
        int gx, cx;
        if (!ghost_choice(sx, i, P.n[0], P.bc[0], P.bc[1], gx, cx)) continue;
        // Face maps applied in ascending dimension (SetBC's face order).
        T a = v0, b = v1;
        if (sx) {
          a = bc_map<T>(cx, a);
          b = bc_map<T>(cx, b);
        }
        if (sy) {
          a = bc_map<T>(cy, a);
          b = bc_map<T>(cy, b);
        }
        if (sz) {
          a = bc_map<T>(cz, a);
          b = bc_map<T>(cz, b);
        }
        const int64_t c = cidx(P, gx, gy, D == 3 ? gz : 0);
        q0[c] = a;
        q1[c] = b;
      }
    }
  }
}

template <class T, int D>
__device__ __forceinline__ void load_stencil(const DevPatch& P, const T* __restrict__ q0,
                                             const T* __restrict__ q1, int64_t c,
                                             Problem::Stencil<T, D>& s) {
  const int64_t st[3] = {1, P.sy, P.sz};
  s.pc = q0[c];
  s.mc = q1[c];
#pragma unroll
  for (int d = 0; d < D; ++d) {
    s.pm[d] = q0[c - st[d]];
    s.pp[d] = q0[c + st[d]];
    s.mm[d] = q1[c - st[d]];
    s.mp[d] = q1[c + st[d]];
  }
}

__device__ __forceinline__ bool near_boundary(const DevPatch& P, int i, int j, int k, int D) {
  bool b = (i == 1) | (i == P.n[0]) | (j == 1) | (j == P.n[1]);
  if (D == 3) b = b | (k == 1) | (k == P.n[2]);
  return b;
}

// ---- per-cell bodies ---------------------------------------------------------

// One cell of RelaxGrid (problem.f90:192-213 / 485-516), in place on q, with
// SetGhost(level, ipass) for physical faces.
template <class T, int D>
__device__ __forceinline__ void relax_cell(const DevPatch& P, int i, int j, int k) {
  T* q0 = fld<T>(P.q[0]);
  T* q1 = fld<T>(P.q[1]);
  const T* f0 = fld<T>(P.f[0]);
  const T* f1 = fld<T>(P.f[1]);
  const int64_t c = cidx(P, i, j, k);
  Problem::Stencil<T, D> s;
  load_stencil<T, D>(P, q0, q1, c, s);
  T phi, mu;
  if (P.delta)
    Problem::RelaxCell<T, D, true>(s, f0[c], f1[c], T(P.tmp1), T(P.tmp2), T(P.tmp3), T(P.alpha),
                                   phi, mu, fld<T>(P.bs)[c]);
  else
    Problem::RelaxCell<T, D>(s, f0[c], f1[c], T(P.tmp1), T(P.tmp2), T(P.tmp3), T(P.alpha), phi,
                             mu);
  q0[c] = phi;
  q1[c] = mu;
  if (P.wt && near_boundary(P, i, j, k, D)) write_through<T, D>(P, q0, q1, i, j, k, phi, mu);
}

// Operator at one cell from its stencil, in the patch's form.
template <class T, int D>
__device__ __forceinline__ void operator_at(const DevPatch& P, const Problem::Stencil<T, D>& s,
                                            int64_t c, T& o0, T& o1) {
  if (P.delta)
    Problem::OperatorCell<T, D, true>(s, T(P.tmp1), T(P.tmp2), T(P.alpha), o0, o1,
                                      fld<T>(P.bs)[c]);
  else
    Problem::OperatorCell<T, D>(s, T(P.tmp1), T(P.tmp2), T(P.alpha), o0, o1);
}

// Residual rf = f - Operator(q) at one cell (afas:799-840).
template <class T, int D>
__device__ __forceinline__ void residual_cell(const DevPatch& P, const T* q0, const T* q1,
                                              const T* f0, const T* f1, int64_t c, T& r0,
                                              T& r1) {
  Problem::Stencil<T, D> s;
  load_stencil<T, D>(P, q0, q1, c, s);
  T o0, o1;
  operator_at<T, D>(P, s, c, o0, o1);
  r0 = f0[c] - o0;
  r1 = f1[c] - o1;
}

// RestrictSolution (afas:600-644) of the coarse cell (ic,jc,kc) of child C
// into parent P, + the parent's SetGhost(level-1, 0) for physical faces +
// GetCoarseGhostPoints (boundary.f90:1203-1269): the parent solution and its
// snapshot qs (the children's qc) are both written.
// TC / TP: value types of the child and the parent (equal in the FP64 path;
// in the mixed path the child may be FP32 over an FP64 parent).  Restriction
// runs in the child's precision; the stored value converts exactly upward.
template <class TC, class TP, int D>
__device__ __forceinline__ void restrict_cell(const DevPatch& C, const DevPatch& P, int ic, int jc,
                                              int kc) {
  const int i = 2 * ic, j = 2 * jc, k = 2 * kc;
  TP val[2];
#pragma unroll
  for (int v = 0; v < 2; ++v) {
    const TC* a = fld<TC>(mid_state(C)[v]);
    if (D == 2) {
      val[v] = TP(TC(0.25) * (a[cidx(C, i, j, 0)] + a[cidx(C, i - 1, j, 0)] +
                              a[cidx(C, i, j - 1, 0)] + a[cidx(C, i - 1, j - 1, 0)]));
    } else {
      val[v] = TP(TC(0.125) * (a[cidx(C, i, j, k)] + a[cidx(C, i - 1, j, k)] +
                               a[cidx(C, i, j - 1, k)] + a[cidx(C, i - 1, j - 1, k)] +
                               a[cidx(C, i, j, k - 1)] + a[cidx(C, i - 1, j, k - 1)] +
                               a[cidx(C, i, j - 1, k - 1)] + a[cidx(C, i - 1, j - 1, k - 1)]));
    }
  }
  const int pi = C.off[0] + ic, pj = C.off[1] + jc, pk = (D == 3) ? C.off[2] + kc : 0;
  const int64_t pc = cidx(P, pi, pj, pk);
  TP* pq0 = fld<TP>(P.q[0]);
  TP* pq1 = fld<TP>(P.q[1]);
  TP* ps0 = fld<TP>(P.qs[0]);
  TP* ps1 = fld<TP>(P.qs[1]);
  pq0[pc] = val[0];
  pq1[pc] = val[1];
  ps0[pc] = val[0];
  ps1[pc] = val[1];
  if (P.wt && near_boundary(P, pi, pj, pk, D)) {
    write_through<TP, D>(P, pq0, pq1, pi, pj, pk, val[0], val[1]);
    write_through<TP, D>(P, ps0, ps1, pi, pj, pk, val[0], val[1]);
  }
  if (P.delta) {
    // Correction form: the coarse base is the restriction of the fine base.
    const TC* b = fld<TC>(C.bs);
    if (D == 2)
      fld<TP>(P.bs)[pc] = TP(TC(0.25) * (b[cidx(C, i, j, 0)] + b[cidx(C, i - 1, j, 0)] +
                                         b[cidx(C, i, j - 1, 0)] + b[cidx(C, i - 1, j - 1, 0)]));
    else
      fld<TP>(P.bs)[pc] =
          TP(TC(0.125) * (b[cidx(C, i, j, k)] + b[cidx(C, i - 1, j, k)] + b[cidx(C, i, j - 1, k)] +
                          b[cidx(C, i - 1, j - 1, k)] + b[cidx(C, i, j, k - 1)] +
                          b[cidx(C, i - 1, j, k - 1)] + b[cidx(C, i, j - 1, k - 1)] +
                          b[cidx(C, i - 1, j - 1, k - 1)]));
  }
}

// CoarseLoadingFunction (afas:646-714) at one coarse cell:
//   parent%f(mb) = Restriction(f - Operator(q)) + Operator(qc, h = parent%dx)
template <class TC, class TP, int D>
__device__ __forceinline__ void coarse_load_cell(const DevPatch& C, const DevPatch& P, int ic,
                                                 int jc, int kc) {
  const TC* q0 = fld<TC>(mid_state(C)[0]);
  const TC* q1 = fld<TC>(mid_state(C)[1]);
  const TC* f0 = fld<TC>(C.f[0]);
  const TC* f1 = fld<TC>(C.f[1]);
  const int i = 2 * ic, j = 2 * jc, k = 2 * kc;
  // Restriction of rf: children in the reference's summation order.
  const int nch = (D == 2) ? 4 : 8;
  TC s0 = TC(0), s1 = TC(0);
#pragma unroll
  for (int ch = 0; ch < nch; ++ch) {
    const int ii = i - (ch & 1), jj = j - ((ch >> 1) & 1), kk = (D == 3) ? k - (ch >> 2) : 0;
    TC r0, r1;
    residual_cell<TC, D>(C, q0, q1, f0, f1, cidx(C, ii, jj, kk), r0, r1);
    if (ch == 0) {
      s0 = r0;
      s1 = r1;
    } else {
      s0 = s0 + r0;
      s1 = s1 + r1;
    }
  }
  const TC w = (D == 2) ? TC(0.25) : TC(0.125);
  const TP R0 = TP(w * s0), R1 = TP(w * s1);
  const int pi = C.off[0] + ic, pj = C.off[1] + jc, pk = (D == 3) ? C.off[2] + kc : 0;
  const int64_t pc = cidx(P, pi, pj, pk);
  Problem::Stencil<TP, D> s;
  load_stencil<TP, D>(P, fld<TP>(P.qs[0]), fld<TP>(P.qs[1]), pc, s);
  TP o0, o1;
  operator_at<TP, D>(P, s, pc, o0, o1);
  fld<TP>(P.f[0])[pc] = R0 + o0;
  fld<TP>(P.f[1])[pc] = R1 + o1;
}

template <class T>
__device__ __forceinline__ T lin_x(bool even, T a, T b) {
  return even ? T(3) * a + b : a + T(3) * b;
}

// CorrectFine with BiLin/TriLinProlongationP1 (afas:842-963,
// gridutilities.f90:137-175, 474-529) at the fine cell (I,J,K):
// q += P(parent%q - qc); the ghost ring is refreshed by write-through (the
// reference's SetGhost(level, 0) overwrites the prolongated ring, afas:515).
// The correction e = parent%q - qc is formed and prolongated in the parent's
// precision and added in the child's.
template <class TC, class TP, int D>
__device__ __forceinline__ void correct_cell(const DevPatch& C, const DevPatch& P, int I, int J,
                                             int K) {
  const TP* pq0 = fld<TP>(P.q[0]);
  const TP* pq1 = fld<TP>(P.q[1]);
  const TP* ps0 = fld<TP>(P.qs[0]);
  const TP* ps1 = fld<TP>(P.qs[1]);
  TC* q0 = fld<TC>(mid_state(C)[0]);
  TC* q1 = fld<TC>(mid_state(C)[1]);
  const int m = I >> 1, n = J >> 1, p = K >> 1;
  const bool ex = (I & 1) == 0, ey = (J & 1) == 0, ez = (K & 1) == 0;
  TP corr[2];
#pragma unroll
  for (int v = 0; v < 2; ++v) {
    const TP* pq = v ? pq1 : pq0;
    const TP* ps = v ? ps1 : ps0;
    auto e = [&](int a, int b, int c) -> TP {
      const int64_t x = cidx(P, C.off[0] + a, C.off[1] + b, D == 3 ? C.off[2] + c : 0);
      return pq[x] - ps[x];
    };
    if (D == 2) {
      const TP b0 = lin_x<TP>(ex, e(m, n, 0), e(m + 1, n, 0));
      const TP b1 = lin_x<TP>(ex, e(m, n + 1, 0), e(m + 1, n + 1, 0));
      corr[v] = lin_x<TP>(ey, b0, b1) / TP(16);
    } else {
      const TP b00 = lin_x<TP>(ex, e(m, n, p), e(m + 1, n, p));
      const TP b10 = lin_x<TP>(ex, e(m, n + 1, p), e(m + 1, n + 1, p));
      const TP b01 = lin_x<TP>(ex, e(m, n, p + 1), e(m + 1, n, p + 1));
      const TP b11 = lin_x<TP>(ex, e(m, n + 1, p + 1), e(m + 1, n + 1, p + 1));
      const TP c0 = lin_x<TP>(ey, b00, b10);
      const TP c1 = lin_x<TP>(ey, b01, b11);
      corr[v] = lin_x<TP>(ez, c0, c1) / TP(64);
    }
  }
  const int64_t c = cidx(C, I, J, K);
  const TC a0 = q0[c] + TC(corr[0]);
  const TC a1 = q1[c] + TC(corr[1]);
  q0[c] = a0;
  q1[c] = a1;
  if (C.wt && near_boundary(C, I, J, K, D)) write_through<TC, D>(C, q0, q1, I, J, K, a0, a1);
}

// ---- reductions --------------------------------------------------------------

// Deterministic block sum of a double (fixed shuffle tree + fixed smem
// order).  Any block shape whose size is a multiple of 32 and at most 1024.
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthreads = blockDim.x * blockDim.y * blockDim.z;
  const int lane = tid & 31, warp = tid >> 5;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (tid == 0) {
    for (int w = 0; w < nthreads / 32; ++w) s += red[w];
  }
  __syncthreads();
  return s;  // valid in thread 0
}

// Second stage of a two-stage reduction: the last CTA to finish sums the
// per-CTA partials in index order.  Returns true in thread 0 of that CTA
// with the total in `total`.
__device__ __forceinline__ bool last_block_total(double mine, double* partials,
                                                 uint32_t* ticket, int nblocks,
                                                 double& total) {
  __shared__ bool is_last;
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthreads = blockDim.x * blockDim.y * blockDim.z;
  if (tid == 0) {
    partials[blockIdx.x] = mine;
    __threadfence();
    const uint32_t t = atomicAdd(ticket, 1u);
    is_last = (t == (uint32_t)nblocks - 1u);
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
  double s = 0.0;
  for (int b = tid; b < nblocks; b += nthreads) s += ((volatile double*)partials)[b];
  const double tot = block_sum(s);
  if (tid == 0) {
    total = tot;
    *ticket = 0u;
    return true;
  }
  return false;
}

// ---- tile bodies ---------------------------------------------------------------
//
// One function per kernel that processes one Item (tile) of its work list.
// The grid kernels below run one tile per CTA; the batch kernels (batch.cuh)
// run the same bodies in a grid-stride loop over a device-resident list.
// Inactive patches (finished or idle batch slots) are skipped whole, which is
// uniform per CTA.

// RelaxGrid (one colour pass) + SetGhost(level, ipass) for physical faces.
// color 0 = ipass 1 = cells with even i+j(+k); color 1 = ipass 2.
template <class T, int D>
__device__ __forceinline__ void relax_item(const DevPatch* __restrict__ PT, const Item it,
                                           int color) {
  const DevPatch P = PT[it.patch];  // by value: fields stay in registers
  if (!P.active) return;
  const int j = it.ty * TILE_Y + threadIdx.y + 1;
  const int k = (D == 3) ? it.tz + 1 : 0;
  if (j > P.n[1]) return;
  const int i0 = (it.tx * 32 + threadIdx.x) * 2 + 1;
  const int i = i0 + ((i0 + j + k + color) & 1);
  if (i > P.n[0]) return;
  relax_cell<T, D>(P, i, j, k);
}

// Sum of rf^2 over this thread's cells of a tile (ErrorAFAS's SquareSum).
template <class T, int D>
__device__ __forceinline__ double resid_item(const DevPatch& P, const Item it) {
  const int j = it.ty * TILE_Y + threadIdx.y + 1;
  const int k = (D == 3) ? it.tz + 1 : 0;
  const int i0 = (it.tx * 32 + threadIdx.x) * 2 + 1;
  const T* q0 = fld<T>(P.q[0]);
  const T* q1 = fld<T>(P.q[1]);
  const T* f0 = fld<T>(P.f[0]);
  const T* f1 = fld<T>(P.f[1]);
  double acc = 0.0;
  if (j <= P.n[1]) {
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      const int i = i0 + t;
      if (i <= P.n[0]) {
        T r0, r1;
        residual_cell<T, D>(P, q0, q1, f0, f1, cidx(P, i, j, k), r0, r1);
        acc += (double)r0 * (double)r0 + (double)r1 * (double)r1;
      }
    }
  }
  return acc;
}

template <class TC, class TP, int D>
__device__ __forceinline__ void restrict_item(const DevPatch* __restrict__ PT, const Item it) {
  const DevPatch C = PT[it.patch];
  if (!C.active) return;
  const DevPatch P = PT[C.parent];
  const int jc = it.ty * TILE_Y + threadIdx.y + 1;
  const int kc = (D == 3) ? it.tz + 1 : 0;
  if (jc > C.cn[1]) return;
  const int ic0 = (it.tx * 32 + threadIdx.x) * 2 + 1;
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    const int ic = ic0 + t;
    if (ic > C.cn[0]) break;
    restrict_cell<TC, TP, D>(C, P, ic, jc, kc);
  }
}

template <class TC, class TP, int D>
__device__ __forceinline__ void coarse_load_item(const DevPatch* __restrict__ PT, const Item it) {
  const DevPatch C = PT[it.patch];
  if (!C.active) return;
  const DevPatch P = PT[C.parent];
  const int jc = it.ty * TILE_Y + threadIdx.y + 1;
  const int kc = (D == 3) ? it.tz + 1 : 0;
  if (jc > C.cn[1]) return;
  const int ic0 = (it.tx * 32 + threadIdx.x) * 2 + 1;
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    const int ic = ic0 + t;
    if (ic > C.cn[0]) break;
    coarse_load_cell<TC, TP, D>(C, P, ic, jc, kc);
  }
}

template <class TC, class TP, int D>
__device__ __forceinline__ void correct_item(const DevPatch* __restrict__ PT, const Item it) {
  const DevPatch C = PT[it.patch];
  if (!C.active) return;
  const DevPatch P = PT[C.parent];
  const int J = it.ty * TILE_Y + threadIdx.y + 1;
  const int K = (D == 3) ? it.tz + 1 : 0;
  if (J > C.n[1]) return;
  const int I0 = (it.tx * 32 + threadIdx.x) * 2 + 1;
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    const int I = I0 + t;
    if (I > C.n[0]) break;
    correct_cell<TC, TP, D>(C, P, I, J, K);
  }
}

// GetSourceFunction + UpdateSourceFunction on one level (afas:312-367,
// 427-486): f = Source(qold) + 0.  newstep_only (batches): only masters
// whose new time step starts now; they keep no qold, so qold = q (the
// reference's CopyQToQold just before, lib/bsamroutines.f90:659-661).
template <class T, int D>
__device__ __forceinline__ void source_item(const DevPatch* __restrict__ PT, const Item it,
                                            int newstep_only) {
  const DevPatch P = PT[it.patch];
  if (!P.active || (newstep_only && !P.newstep)) return;
  const int j = it.ty * TILE_Y + threadIdx.y + 1;
  const int k = (D == 3) ? it.tz + 1 : 0;
  if (j > P.n[1]) return;
  const int i0 = (it.tx * 32 + threadIdx.x) * 2 + 1;
  const T* qo = fld<T>(P.qo[0] ? P.qo[0] : P.q[0]);
  T* f0 = fld<T>(P.f[0]);
  T* f1 = fld<T>(P.f[1]);
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    const int i = i0 + t;
    if (i > P.n[0]) break;
    const int64_t c = cidx(P, i, j, k);
    T a, b;
    Problem::SourceCell<T>(qo[c], T(P.alpha), a, b);
    f0[c] = a;
    f1[c] = b;
  }
}

// ---- grid kernels (one tile per CTA) --------------------------------------------

template <class T, int D>
__global__ void __launch_bounds__(BLOCK_THREADS)
    k_relax(const DevPatch* __restrict__ PT, const Item* __restrict__ items, int color) {
  relax_item<T, D>(PT, items[blockIdx.x], color);
}

// ErrorAFAS / L2Error / SquareSum (afas:108-221), errortype 1:
// residual = sqrt(sum rf^2 / (nrvars * ncells)) over the finest level.
template <class T, int D>
__global__ void __launch_bounds__(BLOCK_THREADS)
    k_resid_norm(const DevPatch* __restrict__ PT, const Item* __restrict__ items,
                 double* __restrict__ partials, DevStatus* __restrict__ st, int nitems,
                 double denom, double tol) {
  const Item it = items[blockIdx.x];
  const double bs = block_sum(resid_item<T, D>(PT[it.patch], it));
  double total;
  if (last_block_total(bs, partials, &st->ticket, nitems, total)) {
    const double r = sqrt(total / denom);
    st->sumsq = total;
    st->residual = r;
    st->converged = (r < tol) ? 1 : 0;
  }
}

template <class TC, class TP, int D>
__global__ void __launch_bounds__(BLOCK_THREADS)
    k_restrict(const DevPatch* __restrict__ PT, const Item* __restrict__ items) {
  restrict_item<TC, TP, D>(PT, items[blockIdx.x]);
}

template <class TC, class TP, int D>
__global__ void __launch_bounds__(BLOCK_THREADS)
    k_coarse_load(const DevPatch* __restrict__ PT, const Item* __restrict__ items) {
  coarse_load_item<TC, TP, D>(PT, items[blockIdx.x]);
}

template <class TC, class TP, int D>
__global__ void __launch_bounds__(BLOCK_THREADS)
    k_correct(const DevPatch* __restrict__ PT, const Item* __restrict__ items) {
  correct_item<TC, TP, D>(PT, items[blockIdx.x]);
}

template <class T, int D>
__global__ void __launch_bounds__(BLOCK_THREADS)
    k_source(const DevPatch* __restrict__ PT, const Item* __restrict__ items) {
  source_item<T, D>(PT, items[blockIdx.x], 0);
}

// SetBC (boundary.f90:598-891), preceded by PeriodicBC on periodic faces
// (boundary.f90:76-83, 417-483), for one patch, all ghost cells, any face
// codes: a ghost is written when at least one of the dimensions it lies
// outside of has a physical or periodic face; its value is the face maps of
// those dimensions (ascending; a periodic face maps a value to itself)
// applied to the cell reflected across them (across a periodic face, the
// cell at the other end).
template <class T, int D>
__device__ __forceinline__ void setbc_elem(const DevPatch& P, int64_t g) {
  const int e0 = P.n[0] + 2, e1 = P.n[1] + 2;
  int co[3] = {(int)(g % e0), (int)((g / e0) % e1), D == 3 ? (int)(g / ((int64_t)e0 * e1)) : 0};
  int src[3] = {co[0], co[1], co[2]};
  int codes[3] = {BC_NONE, BC_NONE, BC_NONE};
  bool write = false;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    if (co[d] == 0 && P.bc[2 * d] != BC_NONE) {
      src[d] = P.bc[2 * d] == BC_PERIODIC ? P.n[d] : 1;
      codes[d] = P.bc[2 * d];
      write = true;
    } else if (co[d] == P.n[d] + 1 && P.bc[2 * d + 1] != BC_NONE) {
      src[d] = P.bc[2 * d + 1] == BC_PERIODIC ? 1 : P.n[d];
      codes[d] = P.bc[2 * d + 1];
      write = true;
    }
  }
  if (!write) return;
#pragma unroll
  for (int v = 0; v < 2; ++v) {
    T* q = fld<T>(P.q[v]);
    T val = q[cidx(P, src[0], src[1], src[2])];
#pragma unroll
    for (int d = 0; d < D; ++d)
      if (codes[d] != BC_NONE) val = bc_map<T>(codes[d], val);
    q[cidx(P, co[0], co[1], co[2])] = val;
  }
}

// One patch, one thread per element of its box with ring (ntotal elements).
template <class T, int D>
__global__ void k_setbc(const DevPatch* __restrict__ PT, int patch, int64_t ntotal) {
  const DevPatch P = PT[patch];
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ntotal) return;
  setbc_elem<T, D>(P, g);
}

// The same for a list of patches (blockIdx.y selects the patch; the grid
// strides over its elements).
template <class T, int D>
__global__ void k_setbc_list(const DevPatch* __restrict__ PT, const int* __restrict__ patches) {
  const DevPatch P = PT[patches[blockIdx.y]];
  const int64_t ntotal =
      (int64_t)(P.n[0] + 2) * (P.n[1] + 2) * (D == 3 ? (int64_t)(P.n[2] + 2) : 1);
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < ntotal;
       g += (int64_t)gridDim.x * blockDim.x)
    setbc_elem<T, D>(P, g);
}

// ---- device-side V-cycle loop (MultigridIterations, afas:69-104) -----------

// Start of a MultigridIterations call: no V-cycle done yet.
static __global__ void k_mg_begin(DevStatus* __restrict__ st) {
  st->iters = 0;
  st->converged = 0;
}

// End of one V-cycle: record the residual and decide whether the conditional
// WHILE node of the step graph runs another V-cycle.  Stops at convergence
// (residual < qerrortol), after maxvcycles, on a non-finite residual (the
// host reports it) or when a kernel recorded an error.
static __global__ void k_mg_loop(DevStatus* __restrict__ st, double* __restrict__ trace, int maxv,
                          double tol, cudaGraphConditionalHandle handle) {
  const int it = st->iters + 1;
  st->iters = it;
  const double r = st->residual;
  if (it <= maxv) trace[it - 1] = r;
  const bool conv = r < tol;
  st->converged = conv ? 1 : 0;
  const bool again = !conv && it < maxv && isfinite(r) && st->kerr == 0;
  cudaGraphSetConditional(handle, again ? 1u : 0u);
}

// One of the two sums of Energy2D (problem.f90:330-361) over a 2D patch
// interior: which = 0, sum of Ff(c); which = 1, sum of f1(i) + f1(i-1) +
// f2(j) + f2(j-1) with f1 = (c(i+1) - c(i))^2, f2 = (c(j+1) - c(j))^2 (the
// ghost ring supplies the outer differences).
template <class T>
__global__ void __launch_bounds__(BLOCK_THREADS)
    k_energy2(const DevPatch* __restrict__ PT, const Item* __restrict__ items,
              double* __restrict__ partials, DevStatus* __restrict__ st, int nitems, int which) {
  const Item it = items[blockIdx.x];
  const DevPatch P = PT[it.patch];
  const int j = it.ty * TILE_Y + threadIdx.y + 1;
  const int i0 = (it.tx * 32 + threadIdx.x) * 2 + 1;
  const T* c = fld<T>(P.q[0]);
  auto C = [&](int i, int jj) { return (double)c[cidx(P, i, jj, 0)]; };
  double acc = 0.0;
  if (j <= P.n[1]) {
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      const int i = i0 + t;
      if (i > P.n[0]) break;
      if (which == 0) {
        acc += Problem::Ff(C(i, j), P.alpha);
      } else {
        const double a = C(i + 1, j) - C(i, j), b = C(i, j) - C(i - 1, j);
        const double u = C(i, j + 1) - C(i, j), w = C(i, j) - C(i, j - 1);
        acc += a * a + b * b + u * u + w * w;
      }
    }
  }
  const double bs = block_sum(acc);
  double total;
  if (last_block_total(bs, partials, &st->ticket, nitems, total)) st->esum = total;
}

// h^d * sum(phi) over a patch interior (AfterStep2D/3D integral(1)).
template <class T, int D>
__global__ void __launch_bounds__(BLOCK_THREADS)
    k_mass(const DevPatch* __restrict__ PT, const Item* __restrict__ items,
           double* __restrict__ partials, DevStatus* __restrict__ st, int nitems, double hd) {
  const Item it = items[blockIdx.x];
  const DevPatch P = PT[it.patch];
  const int j = it.ty * TILE_Y + threadIdx.y + 1;
  const int k = (D == 3) ? it.tz + 1 : 0;
  const int i0 = (it.tx * 32 + threadIdx.x) * 2 + 1;
  const T* q0 = fld<T>(P.q[0]);
  double acc = 0.0;
  if (j <= P.n[1]) {
    if (i0 <= P.n[0]) acc += (double)q0[cidx(P, i0, j, k)];
    if (i0 + 1 <= P.n[0]) acc += (double)q0[cidx(P, i0 + 1, j, k)];
  }
  const double bs = block_sum(acc);
  double total;
  if (last_block_total(bs, partials, &st->ticket, nitems, total)) st->mass = hd * total;
}

}  // namespace bsam
