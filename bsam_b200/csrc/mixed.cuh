// mixed.cuh -- FP64 outer loop around an FP32 FAS V-cycle in correction form.
//
// The mixed form keeps an FP64 master of the finest level (q64, f64).  Each
// V-cycle solves for a correction e of q64 on the "twin" patch and the
// levels below it, which hold FP32 values (small levels FP64):
//
//   r64  = f64 - L64(q64)                    FP64 defect (+ its L2 norm)
//   e    = 0,  base = fl32(phi64),  g = fl32(r64)
//   e   <- FAS V-cycle on  L(base + e) - L(base) = g
//   q64 += e                                  FP64 update
//
// Written for the correction, the inner operator's nonlinear part is
// Dfc(base + e) - Dfc(base) = alpha e (3c^2 + 3ce + e^2) (problem_ch.cuh,
// DfcDelta) and every other term is linear in e, so FP32 rounding scales with
// the correction, not with q; the defect enters the FP32 cycle with its full
// relative precision.  The FAS recursion applies unchanged to e, with each
// level's base restricted from the finer one.  Convergence is judged on the
// FP64 defect of q64, exactly as MultigridIterations judges the FP64 form
// (afas:94-101).
#pragma once
#include "kernels.cuh"

namespace bsam {

// Defect of one master tile: ErrorAFAS of q64 (the same norm as
// k_resid_norm) plus the twin's start (e = 0), base and right-hand side.
// Returns this thread's sum of squares.  newstep_only (batches): only masters
// whose time step starts in this iteration.
template <class TW, int D>
__device__ __forceinline__ double defect_item(const DevPatch* __restrict__ PT, const Item it,
                                              int newstep_only) {
  const DevPatch M = PT[it.patch];
  if (!M.active || (newstep_only && !M.newstep)) return 0.0;
  const DevPatch W = PT[M.twin];
  const int j = it.ty * TILE_Y + threadIdx.y + 1;
  const int k = (D == 3) ? it.tz + 1 : 0;
  const int i0 = (it.tx * 32 + threadIdx.x) * 2 + 1;
  const double* q0 = fld<double>(M.q[0]);
  const double* q1 = fld<double>(M.q[1]);
  const double* f0 = fld<double>(M.f[0]);
  const double* f1 = fld<double>(M.f[1]);
  TW* e0 = fld<TW>(W.q[0]);
  TW* e1 = fld<TW>(W.q[1]);
  double acc = 0.0;
  if (j <= M.n[1]) {
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      const int i = i0 + t;
      if (i > M.n[0]) break;
      const int64_t c = cidx(M, i, j, k);
      double r0, r1;
      residual_cell<double, D>(M, q0, q1, f0, f1, c, r0, r1);
      acc += r0 * r0 + r1 * r1;
      const int64_t cw = cidx(W, i, j, k);
      fld<TW>(W.f[0])[cw] = TW(r0);
      fld<TW>(W.f[1])[cw] = TW(r1);
      fld<TW>(W.bs)[cw] = TW(q0[c]);
      e0[cw] = TW(0);
      e1[cw] = TW(0);
      if (W.wt && near_boundary(W, i, j, k, D))
        write_through<TW, D>(W, e0, e1, i, j, k, TW(0), TW(0));
    }
  }
  return acc;
}

// q64 += e on the interior of one master tile; ghosts by write-through.
template <class TW, int D>
__device__ __forceinline__ void update_item(const DevPatch* __restrict__ PT, const Item it) {
  const DevPatch M = PT[it.patch];
  if (!M.active) return;
  const DevPatch W = PT[M.twin];
  const int j = it.ty * TILE_Y + threadIdx.y + 1;
  const int k = (D == 3) ? it.tz + 1 : 0;
  if (j > M.n[1]) return;
  const int i0 = (it.tx * 32 + threadIdx.x) * 2 + 1;
  double* q0 = fld<double>(M.q[0]);
  double* q1 = fld<double>(M.q[1]);
  const TW* e0 = fld<TW>(W.q[0]);
  const TW* e1 = fld<TW>(W.q[1]);
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    const int i = i0 + t;
    if (i > M.n[0]) break;
    const int64_t c = cidx(M, i, j, k), cw = cidx(W, i, j, k);
    const double na = q0[c] + (double)e0[cw];
    const double nb = q1[c] + (double)e1[cw];
    q0[c] = na;
    q1[c] = nb;
    if (M.wt && near_boundary(M, i, j, k, D)) write_through<double, D>(M, q0, q1, i, j, k, na, nb);
  }
}

// Defect kernel over the masters' tiles, with the FP64 norm in d_status.
template <class TW, int D>
__global__ void __launch_bounds__(BLOCK_THREADS)
    k_defect(const DevPatch* __restrict__ PT, const Item* __restrict__ items,
             double* __restrict__ partials, DevStatus* __restrict__ st, int nitems,
             double denom, double tol) {
  const double bs = block_sum(defect_item<TW, D>(PT, items[blockIdx.x], 0));
  double total;
  if (last_block_total(bs, partials, &st->ticket, nitems, total)) {
    const double r = sqrt(total / denom);
    st->sumsq = total;
    st->residual = r;
    st->converged = (r < tol) ? 1 : 0;
  }
}

template <class TW, int D>
__global__ void __launch_bounds__(BLOCK_THREADS)
    k_update(const DevPatch* __restrict__ PT, const Item* __restrict__ items) {
  update_item<TW, D>(PT, items[blockIdx.x]);
}

}  // namespace bsam
