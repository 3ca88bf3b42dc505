// fused2.cuh -- a whole 2D smoothing stage per shared-memory tile.
//
// LevelRelax (afas:523-547) makes 2*nu colour passes over a level, each
// followed by SetGhost.  Done as one launch per pass, every pass streams the
// level's q, f (and the correction form's base) through HBM again.  Here one
// CTA brings a TX x TY tile of the level with a halo of H = 4 cells into
// shared memory (one TMA tensor copy per field), runs all 2*nu <= 4 passes
// there -- pass p on the tile grown by 2*nu-1-p cells, so that every cell it
// reads from pass p-1 is exact -- and writes the tile's interior back once:
// HBM traffic per stage is about one read of (phi, mu, f1, f2[, base]) and
// one write of (phi, mu), plus the halo.
//
// Every cell update is the same per-cell code in the same order of passes as
// RelaxGrid2D; cells in a tile's halo are recomputed redundantly from the
// same inputs, so the result is bit-identical to the per-pass kernels.
// Physical ghosts inside the tile are refreshed after each update exactly as
// the per-pass write-through does (in a 5-point pass a face ghost is read only
// by its own mirror cell, the one that writes it).  The stage reads one state
// buffer and writes the other (q -> qb before the coarse-grid correction,
// qb -> q after it), so no tile reads a neighbour's already-smoothed cells.
//
// Thread layout: warp w takes rows w, w + 8, ...; lane l the cell pair
// (2l, 2l+1) of a row, of which it updates the one of the pass's colour.
// TX = 56 keeps the widest pass (TX + 6 cells) within 31 pairs.
#pragma once
#include "kernels.cuh"
#include "smooth_fused.cuh"

namespace bsam {

template <class T>
struct Fused2 {
  static constexpr int TX = 56;
  static constexpr int TY = sizeof(T) == 4 ? 32 : 16;
  static constexpr int H = 4;  // halo: supports 2*nu <= 4 passes
  static constexpr int RX = TX + 2 * H;  // 64: 256 / 512-byte shared rows
  static constexpr int RY = TY + 2 * H;
  static constexpr int PLANE = RX * RY;
  static constexpr int NF = 5;  // phi, mu, f1, f2, base
  static constexpr int THREADS = 256;
  static constexpr int WARPS = THREADS / 32;
  static constexpr size_t SMEM = sizeof(T) * NF * PLANE;
  // Shared bytes of a launch: the base plane only for correction-form levels.
  static constexpr size_t smem(bool delta) { return sizeof(T) * (delta ? NF : NF - 1) * PLANE; }
  static_assert((sizeof(T) * PLANE) % 128 == 0, "field planes stay 128-byte aligned");
};

// Tiled 2D tensor copy global -> shared (no multicast).  x * sizeof(T) is a
// multiple of 16 bytes at every call site: x = tile origin (a multiple of 56
// cells) - 3 + lead, with lead = 31 (FP32) or 15 (FP64).
__device__ __forceinline__ void tma_load_2d(void* dst, const void* tmap, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, "
      "{%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(tmap), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Bounded wait on an mbarrier phase by one thread, sleeping between polls
// (32 ns doubling to 512 ns).  Returns false after `limit` polls.
__device__ __forceinline__ bool mbar_wait_backoff(uint64_t* b, uint32_t parity, uint32_t limit) {
  uint32_t ns = 32;
  for (uint32_t it = 0; it < limit; ++it) {
    if (mbar_try_wait(b, parity)) return true;
    __nanosleep(ns);
    if (ns < 512) ns <<= 1;
  }
  return false;
}

// Ghost images of the updated cell (i,j) inside the shared tile: the face
// maps of SetBC2D (boundary.f90:661-738), as write_through applies them.
template <class T>
__device__ __forceinline__ void smem_ghosts2(const DevPatch& P, T* s0, T* s1, int si, int i,
                                             int j, T v0, T v1) {
  constexpr int RX = Fused2<T>::RX;
  if (i == 1 && P.bc[0] != BC_NONE) {
    s0[si - 1] = bc_map<T>(P.bc[0], v0);
    s1[si - 1] = bc_map<T>(P.bc[0], v1);
  }
  if (i == P.n[0] && P.bc[1] != BC_NONE) {
    s0[si + 1] = bc_map<T>(P.bc[1], v0);
    s1[si + 1] = bc_map<T>(P.bc[1], v1);
  }
  if (j == 1 && P.bc[2] != BC_NONE) {
    s0[si - RX] = bc_map<T>(P.bc[2], v0);
    s1[si - RX] = bc_map<T>(P.bc[2], v1);
  }
  if (j == P.n[1] && P.bc[3] != BC_NONE) {
    s0[si + RX] = bc_map<T>(P.bc[3], v0);
    s1[si + RX] = bc_map<T>(P.bc[3], v1);
  }
}

// CorrectFine (afas:842-963) of the cells of a shared tile: every cell of the
// tile inside the patch's interior takes the bilinear prolongation of the
// parent's q - qs (the change of the coarse solution), the expression of
// correct_block2, so the tile holds what kb_correct2 would have written.
template <class T, class TP>
__device__ __forceinline__ void correct_tile2(const DevPatch& C, const DevPatch& R, T* s0, T* s1,
                                              int gx0, int gy0) {
  constexpr int RX = Fused2<T>::RX, RY = Fused2<T>::RY;
  const TP* pq0 = fld<TP>(R.q[0]);
  const TP* pq1 = fld<TP>(R.q[1]);
  const TP* ps0 = fld<TP>(R.qs[0]);
  const TP* ps1 = fld<TP>(R.qs[1]);
  // Coarse blocks (m, n) whose fine cells 2m + {0, 1}, 2n + {0, 1} meet the
  // tile: the four coarse differences are loaded once per block.
  const int mlo = (gx0 >= 0 ? gx0 : gx0 - 1) / 2, nlo = (gy0 >= 0 ? gy0 : gy0 - 1) / 2;
  const int bw = (gx0 + RX - 1) / 2 - mlo + 1, bh = (gy0 + RY - 1) / 2 - nlo + 1;
  for (int blk = threadIdx.x; blk < bw * bh; blk += blockDim.x) {
    const int m = mlo + blk % bw, n = nlo + blk / bw;
    if (m < 0 || m > C.cn[0] || n < 0 || n > C.cn[1]) continue;
    TP e[2][2][2];  // [component][m + a][n + b]
#pragma unroll
    for (int v = 0; v < 2; ++v) {
      const TP* pq = v ? pq1 : pq0;
      const TP* ps = v ? ps1 : ps0;
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int bb = 0; bb < 2; ++bb) {
          const int64_t x = cidx(R, C.off[0] + m + a, C.off[1] + n + bb, 0);
          e[v][a][bb] = pq[x] - ps[x];
        }
    }
#pragma unroll
    for (int dy = 0; dy < 2; ++dy) {
      const int J = 2 * n + dy, sy = J - gy0;
      if (J < 1 || J > C.n[1] || sy < 0 || sy >= RY) continue;
#pragma unroll
      for (int dx = 0; dx < 2; ++dx) {
        const int I = 2 * m + dx, sx = I - gx0;
        if (I < 1 || I > C.n[0] || sx < 0 || sx >= RX) continue;
        TP corr[2];
#pragma unroll
        for (int v = 0; v < 2; ++v) {
          const TP b0 = lin_x<TP>(dx == 0, e[v][0][0], e[v][1][0]);
          const TP b1 = lin_x<TP>(dx == 0, e[v][0][1], e[v][1][1]);
          corr[v] = lin_x<TP>(dy == 0, b0, b1) / TP(16);
        }
        const int c = sy * RX + sx;
        s0[c] = s0[c] + T(corr[0]);
        s1[c] = s1[c] + T(corr[1]);
      }
    }
  }
}

// RestrictSolution (afas:600-644) of the coarse cells a tile covers, from the
// smoothed tile in shared memory: the parent's q and its snapshot qs (and,
// in the correction form, the parent's base from the fine base), ghosts by
// write-through -- restrict_cell's expressions.  Tiles start at odd global
// indices and have even sizes, so every 2 x 2 block lies in one tile.
template <class T, class TP, bool DELTA>
__device__ __forceinline__ void restrict_tile2(const DevPatch& C, const DevPatch& R, const T* s0,
                                               const T* s1, const T* sbs, int gx0, int gy0) {
  using F = Fused2<T>;
  const int icl = (gx0 + F::H + 1) / 2, jcl = (gy0 + F::H + 1) / 2;
  TP* pq0 = fld<TP>(R.q[0]);
  TP* pq1 = fld<TP>(R.q[1]);
  TP* ps0 = fld<TP>(R.qs[0]);
  TP* ps1 = fld<TP>(R.qs[1]);
  for (int c = threadIdx.x; c < (F::TX / 2) * (F::TY / 2); c += blockDim.x) {
    const int ic = icl + c % (F::TX / 2), jc = jcl + c / (F::TX / 2);
    if (ic > C.cn[0] || jc > C.cn[1]) continue;
    const int si = (2 * jc - gy0) * F::RX + (2 * ic - gx0);  // fine cell (2ic, 2jc)
    const TP v0 = TP(T(0.25) * (s0[si] + s0[si - 1] + s0[si - F::RX] + s0[si - 1 - F::RX]));
    const TP v1 = TP(T(0.25) * (s1[si] + s1[si - 1] + s1[si - F::RX] + s1[si - 1 - F::RX]));
    const int pi = C.off[0] + ic, pj = C.off[1] + jc;
    const int64_t pc = cidx(R, pi, pj, 0);
    pq0[pc] = v0;
    pq1[pc] = v1;
    ps0[pc] = v0;
    ps1[pc] = v1;
    if (R.wt && near_boundary(R, pi, pj, 0, 2)) {
      write_through<TP, 2>(R, pq0, pq1, pi, pj, 0, v0, v1);
      write_through<TP, 2>(R, ps0, ps1, pi, pj, 0, v0, v1);
    }
    if constexpr (DELTA)
      if (R.delta)
        fld<TP>(R.bs)[pc] =
            TP(T(0.25) * (sbs[si] + sbs[si - 1] + sbs[si - F::RX] + sbs[si - 1 - F::RX]));
  }
}

// dir 0: q -> qb (pre-smoothing); dir 1: qb -> q (post-smoothing).
// P.tmaps: 2D maps of q0, q1, qb0, qb1, f0, f1, bs (box RX x RY).
// A copy that has not landed after kWaitPolls polls sets *err and ends the
// launch for this CTA.  DELTA: every record of the list is a correction-form
// level (the mixed form's working levels), with a base field.
// upd (post-smoothing of the mixed form's finest working level): the smoothed
// correction e is not stored; the tile's cells apply it to the FP64 master
// instead, q64 += e with the master's ghosts by write-through -- the update of
// mixed.cuh (update_item), expression for expression, done here while e is in
// shared memory.  Every CTA writes only its own tile's cells of the master,
// which nothing else in the launch reads.
// corr (post-smoothing): the coarse-grid correction is applied to the tile
// after it lands (correct_tile2, then the physical face ghosts the passes
// read), instead of by a kb_correct2 launch before the stage.
// restr (pre-smoothing): the tile's coarse cells are restricted into the
// parent from shared memory (restrict_tile2), instead of by a kb_restrict
// launch after the stage.
// Four CTAs per SM (the shared tile allows four): the register cap this
// implies costs a few spilled values outside the passes; without it the
// kernel takes 80 registers and three CTAs per SM, which measured slower.
template <class T, bool DELTA>
__global__ void __launch_bounds__(Fused2<T>::THREADS, 4)
    kb_smooth2(const DevPatch* __restrict__ PT, const Item* __restrict__ items,
               const int* __restrict__ count, int dir, int nu, int upd, int corr,
               int restr, int* __restrict__ err) {
  using F = Fused2<T>;
  extern __shared__ __align__(1024) unsigned char smem2_raw[];
  __shared__ __align__(8) uint64_t bar;
  T* s0 = reinterpret_cast<T*>(smem2_raw);
  T* s1 = s0 + F::PLANE;
  T* sf0 = s1 + F::PLANE;
  T* sf1 = sf0 + F::PLANE;
  T* sbs = sf1 + F::PLANE;
  const int n = *count;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int npass = 2 * nu;
  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  uint32_t phase = 0;
  for (int b = blockIdx.x; b < n; b += gridDim.x) {
    const Item it = items[b];
    const DevPatch P = PT[it.patch];
    if (!P.active) continue;  // uniform per CTA
    const int gx0 = it.tx * F::TX + 1 - F::H;  // global i of shared column 0
    const int gy0 = it.ty * F::TY + 1 - F::H;  // global j of shared row 0
    const int lead = 128 / (int)sizeof(T) - 1;
    if (tid == 0) {
      const CUtensorMapOpaque* maps = static_cast<const CUtensorMapOpaque*>(P.tmaps);
      const int m0 = dir == 0 ? 0 : 2;
      const uint32_t plane = (uint32_t)(sizeof(T) * F::PLANE);
      fence_proxy_async_smem();  // earlier generic accesses to the tile come first
      mbar_arrive_expect_tx(&bar, plane * (DELTA ? 5u : 4u));
      const int x = gx0 + lead;  // column of element (gx0, *) from the allocation start
      tma_load_2d(s0, &maps[m0], x, gy0, &bar);
      tma_load_2d(s1, &maps[m0 + 1], x, gy0, &bar);
      tma_load_2d(sf0, &maps[4], x, gy0, &bar);
      tma_load_2d(sf1, &maps[5], x, gy0, &bar);
      if (DELTA) tma_load_2d(sbs, &maps[6], x, gy0, &bar);
    }
    // One thread polls (with back-off, so that the waiting CTA takes no issue
    // slots from the CTAs computing beside it); after the barrier every
    // thread observes the completed phase itself.
    bool ok = true;
    if (tid == 0) ok = mbar_wait_backoff(&bar, phase, kWaitPolls);
    ok = __syncthreads_and(ok);
    if (ok && tid != 0) (void)mbar_try_wait(&bar, phase);
    phase ^= 1u;
    if (!ok) {
      if (tid == 0) atomicExch(err, kErrTmaTimeout);
      break;
    }
    const int n0 = P.n[0], n1 = P.n[1];
    if (corr && P.parent >= 0) {
      const DevPatch R = PT[P.parent];
      if (P.pprec == PREC_F32) correct_tile2<T, float>(P, R, s0, s1, gx0, gy0);
      else correct_tile2<T, double>(P, R, s0, s1, gx0, gy0);
      __syncthreads();
      // Face ghosts of the corrected boundary cells, for the cells whose
      // neighbours lie in the tile (the passes read no others).
      if (P.wt)
        for (int c = tid; c < F::PLANE; c += F::THREADS) {
          const int sx = c % F::RX, sy = c / F::RX;
          if (sx < 1 || sx > F::RX - 2 || sy < 1 || sy > F::RY - 2) continue;
          const int i = gx0 + sx, j = gy0 + sy;
          if (i < 1 || i > n0 || j < 1 || j > n1) continue;
          if (i == 1 || i == n0 || j == 1 || j == n1) smem_ghosts2<T>(P, s0, s1, c, i, j, s0[c], s1[c]);
        }
      __syncthreads();
    }
    T* o0 = fld<T>(dir == 0 ? P.qb[0] : P.q[0]);
    T* o1 = fld<T>(dir == 0 ? P.qb[1] : P.q[1]);
    const T tmp1 = T(P.tmp1), tmp2 = T(P.tmp2), tmp3 = T(P.tmp3), alpha = T(P.alpha);
    for (int p = 0; p < npass; ++p) {
      const int color = p & 1;
      const int grow = npass - 1 - p;
      // Region of this pass in shared coordinates, clipped to the interior.
      const int xa = max(F::H - grow, 1 - gx0), xb = min(F::H + F::TX + grow, n0 + 1 - gx0);
      const int ya = max(F::H - grow, 1 - gy0), yb = min(F::H + F::TY + grow, n1 + 1 - gy0);
      // A warp's rows step by WARPS (even), so the column of the pass's
      // colour in the lane's pair is the same on all of them.
      const int sy0 = ya + warp;
      int sx = xa + 2 * lane;
      if ((gx0 + sx + gy0 + sy0 + color) & 1) ++sx;
      if (sx < xb) {
        const int i = gx0 + sx;
        const bool edge_i = P.wt && (i == 1 || i == n0);
        int si = sy0 * F::RX + sx;
        for (int sy = sy0; sy < yb; sy += F::WARPS, si += F::WARPS * F::RX) {
          problem::Stencil<T, 2> st;
          st.pc = s0[si];
          st.mc = s1[si];
          st.pm[0] = s0[si - 1];
          st.pp[0] = s0[si + 1];
          st.mm[0] = s1[si - 1];
          st.mp[0] = s1[si + 1];
          st.pm[1] = s0[si - F::RX];
          st.pp[1] = s0[si + F::RX];
          st.mm[1] = s1[si - F::RX];
          st.mp[1] = s1[si + F::RX];
          T phi, mu;
          if constexpr (DELTA)
            problem::RelaxCell<T, 2, true>(st, sf0[si], sf1[si], tmp1, tmp2, tmp3, alpha, phi,
                                           mu, sbs[si]);
          else
            problem::RelaxCell<T, 2>(st, sf0[si], sf1[si], tmp1, tmp2, tmp3, alpha, phi, mu);
          s0[si] = phi;
          s1[si] = mu;
          const int j = gy0 + sy;
          if (edge_i || (P.wt && (j == 1 || j == n1)))
            smem_ghosts2<T>(P, s0, s1, si, i, j, phi, mu);
        }
      }
      __syncthreads();
    }
    if (upd && P.master >= 0) {
      const DevPatch M = PT[P.master];
      double* m0 = fld<double>(M.q[0]);
      double* m1 = fld<double>(M.q[1]);
      for (int ly = warp; ly < F::TY; ly += F::WARPS) {
        const int j = gy0 + F::H + ly;
        if (j > n1) break;
        const int srow = (F::H + ly) * F::RX + F::H;
        for (int lx = lane; lx < F::TX; lx += 32) {
          const int i = gx0 + F::H + lx;
          if (i > n0) break;
          const int64_t c = cidx(M, i, j, 0);
          const double na = m0[c] + (double)s0[srow + lx];
          const double nb = m1[c] + (double)s1[srow + lx];
          m0[c] = na;
          m1[c] = nb;
          if (M.wt && near_boundary(M, i, j, 0, 2))
            write_through<double, 2>(M, m0, m1, i, j, 0, na, nb);
        }
      }
      __syncthreads();  // the shared tile is refilled for the next item
      continue;
    }
    if (restr && P.parent >= 0) {
      const DevPatch R = PT[P.parent];
      if (P.pprec == PREC_F32) restrict_tile2<T, float, DELTA>(P, R, s0, s1, sbs, gx0, gy0);
      else restrict_tile2<T, double, DELTA>(P, R, s0, s1, sbs, gx0, gy0);
    }
    // Write back the tile's interior cells (warps over rows, lanes along
    // them), ghosts by write-through.
    for (int ly = warp; ly < F::TY; ly += F::WARPS) {
      const int j = gy0 + F::H + ly;
      if (j > n1) break;
      const int srow = (F::H + ly) * F::RX + F::H;
      T* r0 = o0 + (int64_t)j * P.sy;
      T* r1 = o1 + (int64_t)j * P.sy;
      const bool edge_j = P.wt && (j == 1 || j == n1);
      for (int lx = lane; lx < F::TX; lx += 32) {
        const int i = gx0 + F::H + lx;
        if (i > n0) break;
        const T v0 = s0[srow + lx], v1 = s1[srow + lx];
        r0[i] = v0;
        r1[i] = v1;
        if (edge_j || (P.wt && (i == 1 || i == n0)))
          write_through<T, 2>(P, o0, o1, i, j, 0, v0, v1);
      }
    }
    __syncthreads();  // the shared tile is refilled for the next item
  }
}

}  // namespace bsam
