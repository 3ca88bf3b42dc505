// regrid.cuh -- the device side of regridding: cell tagging and the
// initial state of a new refined patch.
//
//   k_errflags   SetErrFlagsUser2D/3D (problem.f90:135-163, 425-452): a cell is
//                flagged where the undivided central gradient of c = q(...,1)
//                exceeds the level's tolerance.
//   k_init_mc    InitFields (lib/bsamroutines.f90:1685-1772) for mbc = 1: the
//                child's q on (0:mx+1)^d is the mass-corrected linear
//                prolongation (Bi/TriLinProlongationP1MC,
//                gridutilities.f90:219-279, 588-686) of the parent's q over
//                the child's footprint and its one-cell ring; qold = q.
// The clustering of the flags into new patches (Berger-Rigoutsos, NewSubGrids)
// runs on the host (bsam_host_new_subgrids).
#pragma once
#include "kernels.cuh"

namespace bsam {

// Flags (1:mx)^d of patch P, column-major, one byte per cell.
template <int D>
__device__ void errflags_patch(const DevPatch* __restrict__ PT, int patch, double tol,
                               uint8_t* __restrict__ flags) {
  const DevPatch P = PT[patch];
  const double* c = fld<double>(P.q[0]);
  const int n0 = P.n[0], n1 = P.n[1], n2 = D == 3 ? P.n[2] : 1;
  const int64_t total = (int64_t)n0 * n1 * n2;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % n0) + 1;
    const int j = (int)((e / n0) % n1) + 1;
    const int k = D == 3 ? (int)(e / ((int64_t)n0 * n1)) + 1 : 0;
    double dc[D];
    dc[0] = c[cidx(P, i + 1, j, k)] - c[cidx(P, i - 1, j, k)];
    dc[1] = c[cidx(P, i, j + 1, k)] - c[cidx(P, i, j - 1, k)];
    if (D == 3) dc[D - 1] = c[cidx(P, i, j, k + 1)] - c[cidx(P, i, j, k - 1)];
    flags[e] = Problem::TagCell<D>(dc, tol) ? 1 : 0;
  }
}

template <int D>
__global__ void k_errflags(const DevPatch* __restrict__ PT, int patch, double tol,
                           uint8_t* __restrict__ flags) {
  errflags_patch<D>(PT, patch, tol, flags);
}

// The flags of several patches in one launch: blockIdx.y selects the patch
// and its offset in the concatenated flag array.
struct FlagTask {
  int64_t off;
  int32_t patch, pad_;
};

template <int D>
__global__ void k_errflags_list(const DevPatch* __restrict__ PT, const FlagTask* __restrict__ tasks,
                                double tol, uint8_t* __restrict__ flags) {
  const FlagTask t = tasks[blockIdx.y];
  errflags_patch<D>(PT, t.patch, tol, flags + t.off);
}

// ---- buffering and clustering signatures of a level, on the device ----------
//
// BufferAndList + InflateEdgeTags (lib/bsamroutines.f90:1159-1284) make every
// cell of a level's patches flagged that lies within ibuffer cells (in each
// dimension) of a cell flagged by the tagging, in global index space: the
// union of the buffer boxes of the flagged cells, clipped to each patch
// (a flagged cell whose box stays inside its patch only reaches that patch;
// one whose box crosses the patch's edge reaches every patch of the level it
// overlaps).  Berger-Rigoutsos (NewSubGrids, GetSignatures, GridFlagRatio,
// 1352-1579) then only counts flagged cells in boxes and slabs of a patch,
// which an inclusive summed-area table answers with 2^d lookups.

// A patch of the level: its cells' offset in the level's arrays, its extent
// and the global index of its first cell.
struct LevelPatch {
  int64_t off;
  int32_t n[3], g0[3];
};

// Flag of the cell at global index (gi, gj, gk) of the level, 0 outside its
// patches.  `self` is tried first (the common case: the cell's own patch).
template <int D>
__device__ __forceinline__ uint8_t level_flag(const LevelPatch* __restrict__ lp, int np, int self,
                                              const uint8_t* __restrict__ in, int gi, int gj,
                                              int gk) {
  for (int t = -1; t < np; ++t) {
    const int q = t < 0 ? self : t;
    if (t == self) continue;
    const LevelPatch& L = lp[q];
    const int i = gi - L.g0[0], j = gj - L.g0[1], k = D == 3 ? gk - L.g0[2] : 0;
    if (i < 0 || i >= L.n[0] || j < 0 || j >= L.n[1] || (D == 3 && (k < 0 || k >= L.n[2])))
      continue;
    return in[L.off + i + (int64_t)L.n[0] * (j + (int64_t)L.n[1] * k)];
  }
  return 0;
}

// The buffered flags of every patch of a level (blockIdx.y selects the patch).
template <int D>
__global__ void k_buffer_list(const LevelPatch* __restrict__ lp, int np, int ib,
                              const uint8_t* __restrict__ in, uint8_t* __restrict__ out) {
  const int p = blockIdx.y;
  const LevelPatch L = lp[p];
  const int64_t total = (int64_t)L.n[0] * L.n[1] * (D == 3 ? L.n[2] : 1);
  const int kb = D == 3 ? ib : 0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % L.n[0]), j = (int)((e / L.n[0]) % L.n[1]);
    const int k = D == 3 ? (int)(e / ((int64_t)L.n[0] * L.n[1])) : 0;
    // Cells whose whole neighbourhood lies in the patch read it directly.
    const bool inner = i - ib >= 0 && i + ib < L.n[0] && j - ib >= 0 && j + ib < L.n[1] &&
                       (D == 2 || (k - kb >= 0 && k + kb < L.n[2]));
    uint8_t f = 0;
    for (int dk = -kb; dk <= kb && !f; ++dk)
      for (int dj = -ib; dj <= ib && !f; ++dj)
        for (int di = -ib; di <= ib && !f; ++di) {
          if (inner)
            f = in[L.off + (i + di) + (int64_t)L.n[0] * ((j + dj) + (int64_t)L.n[1] * (k + dk))];
          else
            f = level_flag<D>(lp, np, p, in, L.g0[0] + i + di, L.g0[1] + j + dj,
                              D == 3 ? L.g0[2] + k + dk : 0);
        }
    out[L.off + e] = f ? 1 : 0;
  }
}

// Inclusive summed-area table of each patch's flags (a CTA per patch): sums
// along x, then y, then z.  Along x a warp takes a line, 32 cells at a time,
// with a warp-wide scan and the carry from the previous 32; along y (and z)
// a lane takes a column and loads eight cells ahead of its running sum, so
// that the loads are in flight together.  Integer sums, so the table does
// not depend on the order of the additions.
template <int D>
__global__ void __launch_bounds__(256)
    k_sat_list(const LevelPatch* __restrict__ lp, const uint8_t* __restrict__ in,
               int32_t* __restrict__ sat) {
  constexpr unsigned FULL = 0xffffffffu;
  const LevelPatch L = lp[blockIdx.x];
  const int n0 = L.n[0], n1 = L.n[1], n2 = D == 3 ? L.n[2] : 1;
  int32_t* s = sat + L.off;
  const uint8_t* f = in + L.off;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int line = warp; line < n1 * n2; line += nw) {
    const int64_t b = (int64_t)line * n0;
    int32_t carry = 0;
    for (int i0 = 0; i0 < n0; i0 += 256) {
      int32_t v[8];
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        const int i = i0 + 32 * t + lane;
        v[t] = i < n0 ? (int32_t)f[b + i] : 0;
      }
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        int32_t x = v[t];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int32_t u = __shfl_up_sync(FULL, x, o);
          if (lane >= o) x += u;
        }
        x += carry;
        const int i = i0 + 32 * t + lane;
        if (i < n0) s[b + i] = x;
        carry = __shfl_sync(FULL, x, 31);
      }
    }
  }
  __syncthreads();
  // Column scans along a stride: `cols` columns (count ncol) of `len` cells.
  auto columns = [&](int64_t ncol, int len, int64_t stride, int64_t plane_cols,
                     int64_t plane_stride) {
    for (int64_t c = threadIdx.x; c < ncol; c += blockDim.x) {
      const int64_t base = (c % plane_cols) + (c / plane_cols) * plane_stride;
      int32_t acc = 0;
      for (int j0 = 0; j0 < len; j0 += 8) {
        int32_t v[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) v[t] = j0 + t < len ? s[base + (j0 + t) * stride] : 0;
#pragma unroll
        for (int t = 0; t < 8; ++t) {
          acc += v[t];
          if (j0 + t < len) s[base + (j0 + t) * stride] = acc;
        }
      }
    }
  };
  // y: column i of plane k, cells i + n0 (j + n1 k), j = 0 .. n1 - 1.
  columns((int64_t)n0 * n2, n1, n0, n0, (int64_t)n0 * n1);
  if (D == 3) {
    __syncthreads();
    // z: column (i, j), cells i + n0 j + n0 n1 k, k = 0 .. n2 - 1.
    columns((int64_t)n0 * n1, n2, (int64_t)n0 * n1, (int64_t)n0 * n1, 0);
  }
}

// The linear-prolongation weights of fine index I from coarse (qc) indices
// I >> 1 and (I >> 1) + 1: 3 and 1 for even I, 1 and 3 for odd I.
__device__ __forceinline__ double lin_pair(int I, double a0, double a1) {
  return (I & 1) == 0 ? 3.0 * a0 + a1 : a0 + 3.0 * a1;
}

// The uncorrected prolongation of qc (parent q, footprint + ring) at fine
// cell (I, J[, K]) of the child, I in 0..mx+1: x first, then y, then z, as
// the reference's temporaries b (and c) hold them.
template <int D>
__device__ __forceinline__ double prolong_raw(const DevPatch& C, const DevPatch& R, const double* a,
                                              int I, int J, int K) {
  // qc index k maps to parent index off + k.
  auto A = [&](int x, int y, int z) {
    return a[cidx(R, C.off[0] + x, C.off[1] + y, D == 3 ? C.off[2] + z : 0)];
  };
  const int x = I >> 1, y = J >> 1;
  if (D == 2) {
    const double b0 = lin_pair(I, A(x, y, 0), A(x + 1, y, 0));
    const double b1 = lin_pair(I, A(x, y + 1, 0), A(x + 1, y + 1, 0));
    return ((J & 1) == 0 ? 3.0 * b0 + b1 : b0 + 3.0 * b1) / 16.0;
  }
  const int z = K >> 1;
  double c[2];
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    const double b0 = lin_pair(I, A(x, y, z + t), A(x + 1, y, z + t));
    const double b1 = lin_pair(I, A(x, y + 1, z + t), A(x + 1, y + 1, z + t));
    c[t] = lin_pair(J, b0, b1);
  }
  return ((K & 1) == 0 ? 3.0 * c[0] + c[1] : c[0] + 3.0 * c[1]) / 64.0;
}

// InitFields of child patch `child`: threads over the child's coarse cells
// (0:cmx+1)^d; an interior coarse cell writes its 2^d children with the mass
// correction, a ring coarse cell the children of it that lie in the child's
// ring (0:mx+1)^d, uncorrected.  Then qold = q on the same cells.
template <int D>
__device__ void init_mc(const DevPatch* __restrict__ PT, int child) {
  const DevPatch C = PT[child];
  const DevPatch R = PT[C.parent];
  const int c0 = C.cn[0], c1 = C.cn[1], c2 = D == 3 ? C.cn[2] : 0;
  const int e0 = c0 + 2, e1 = c1 + 2, e2 = D == 3 ? c2 + 2 : 1;
  const int64_t total = (int64_t)e0 * e1 * e2;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(e % e0), l = (int)((e / e0) % e1);
    const int n = D == 3 ? (int)(e / ((int64_t)e0 * e1)) : 0;
    const bool interior = k >= 1 && k <= c0 && l >= 1 && l <= c1 && (D == 2 || (n >= 1 && n <= c2));
#pragma unroll
    for (int v = 0; v < 2; ++v) {
      const double* a = fld<double>(R.q[v]);
      double* q = fld<double>(C.q[v]);
      double* qo = fld<double>(C.qo[v]);
      // The children of coarse cell (k, l[, n]): fine 2k - 1, 2k (etc.).
      double p[8];
      int idx[8][3];
      const int nch = D == 2 ? 4 : 8;
      // Child order of the reference's mass-correction sum: (2k,2l[,2n]),
      // (2k-1,2l,..), (2k,2l-1,..), (2k-1,2l-1,..), then the same at 2n-1.
#pragma unroll
      for (int ch = 0; ch < nch; ++ch) {
        idx[ch][0] = 2 * k - (ch & 1);
        idx[ch][1] = 2 * l - ((ch >> 1) & 1);
        idx[ch][2] = D == 3 ? 2 * n - (ch >> 2) : 0;
      }
      if (interior) {
#pragma unroll
        for (int ch = 0; ch < nch; ++ch) p[ch] = prolong_raw<D>(C, R, a, idx[ch][0], idx[ch][1], idx[ch][2]);
        double s;
        if (D == 2) {
          s = a[cidx(R, C.off[0] + k, C.off[1] + l, 0)] - 0.25 * (p[0] + p[1] + p[2] + p[3]);
        } else {
          s = a[cidx(R, C.off[0] + k, C.off[1] + l, C.off[2] + n)] -
              0.125 * (p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7]);
        }
#pragma unroll
        for (int ch = 0; ch < nch; ++ch) {
          const double val = p[ch] + s;
          const int64_t ci = cidx(C, idx[ch][0], idx[ch][1], idx[ch][2]);
          q[ci] = val;
          qo[ci] = val;
        }
      } else {
        // Ring coarse cell: its children inside (0:mx+1)^d, uncorrected.
#pragma unroll
        for (int ch = 0; ch < nch; ++ch) {
          const int I = idx[ch][0], J = idx[ch][1], K = idx[ch][2];
          if (I < 0 || I > 2 * c0 + 1 || J < 0 || J > 2 * c1 + 1) continue;
          if (D == 3 && (K < 0 || K > 2 * c2 + 1)) continue;
          // A fine cell in the ring of the child: not a child of an interior
          // coarse cell.
          const bool fine_interior = I >= 1 && I <= 2 * c0 && J >= 1 && J <= 2 * c1 &&
                                     (D == 2 || (K >= 1 && K <= 2 * c2));
          if (fine_interior) continue;
          const double val = prolong_raw<D>(C, R, a, I, J, K);
          const int64_t ci = cidx(C, I, J, K);
          q[ci] = val;
          qo[ci] = val;
        }
      }
    }
  }
}

template <int D>
__global__ void k_init_mc(const DevPatch* __restrict__ PT, int child) {
  init_mc<D>(PT, child);
}

// InitFields of several new patches in one launch: blockIdx.y selects the
// child (the children are independent: each reads only its parent).
template <int D>
__global__ void k_init_mc_list(const DevPatch* __restrict__ PT, const int* __restrict__ children) {
  init_mc<D>(PT, children[blockIdx.y]);
}

// Contiguous device-to-device copies in one launch: blockIdx.y selects the
// span (CopyQToQold of every patch, the stash of the refined patches).
struct CopySpan {
  const double* src;
  double* dst;
  int64_t n;
};

__global__ void __launch_bounds__(256) k_copy_spans(const CopySpan* __restrict__ spans) {
  const CopySpan s = spans[blockIdx.y];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < s.n;
       i += (int64_t)gridDim.x * blockDim.x)
    s.dst[i] = s.src[i];
}

// TransferOverlap (lib/bsamroutines.f90:1832-1867): the new grid takes the
// stashed old grid's q on the interior cells both cover, in global indices.
// One TransferOverlap of a regrid: the stashed old grid S (its record by
// value), the new grid `target`, the overlap's extent and its first cell in
// each grid's index space.
struct TransferTask {
  DevPatch S;
  int32_t target;
  int32_t n[3], si[3], ti[3];
};

// The transfers of a regrid in one launch (blockIdx.y selects the task).  Two
// tasks with the same target never overlap: the old grids of a level are
// disjoint.
template <int D>
__global__ void k_transfer_list(const DevPatch* __restrict__ PT,
                                const TransferTask* __restrict__ tasks) {
  const TransferTask& t = tasks[blockIdx.y];
  const DevPatch T = PT[t.target];
  const int n0 = t.n[0], n1 = t.n[1], n2 = D == 3 ? t.n[2] : 1;
  const int64_t total = (int64_t)n0 * n1 * n2;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int a = (int)(e % n0), b = (int)((e / n0) % n1);
    const int c = D == 3 ? (int)(e / ((int64_t)n0 * n1)) : 0;
    const int64_t ts = cidx(T, t.ti[0] + a, t.ti[1] + b, D == 3 ? t.ti[2] + c : 0);
    const int64_t ss = cidx(t.S, t.si[0] + a, t.si[1] + b, D == 3 ? t.si[2] + c : 0);
#pragma unroll
    for (int v = 0; v < 2; ++v) fld<double>(T.q[v])[ts] = fld<double>(t.S.q[v])[ss];
  }
}

}  // namespace bsam
