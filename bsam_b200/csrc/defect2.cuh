// defect2.cuh -- the mixed form's FP64 defect of 2D masters, tiles staged by TMA.
//
// defect_item (mixed.cuh) reads the master's q with a 5-point stencil and f
// straight from global memory, two cells per thread; at a few hundred cells
// per tile those loads stall on memory latency (about 40 % of HBM bandwidth
// measured).  Here one thread issues bulk tensor copies of the tile's q
// (both components, one-cell halo) and f into shared memory, and the CTA
// computes from there.  Tiles, the thread-to-cell mapping, every expression
// and the block reduction are those of defect_item, so each tile's partial
// sum -- and so the residual -- is bit for bit the same.
#pragma once
#include "fused2.cuh"
#include "mixed.cuh"

namespace bsam {

struct Defect2 {
  static constexpr int TX = TILE_X;   // 64: cells of a tile row
  static constexpr int TY = TILE_Y;   // rows of a tile
  // q box: columns i0 - 2 .. i0 + TX + 1 (x * 8 bytes stays a multiple of 16
  // bytes: x = lead + i0 - 2 = 64 tx + 14), rows j0 - 1 .. j0 + TY.
  static constexpr int QX = TX + 4;
  static constexpr int QY = TY + 2;
  static constexpr int QPLANE = QX * QY;
  static constexpr int FPLANE = TX * TY;  // f box: the tile's interior
  // Shared planes start on 128-byte boundaries (TMA destinations).
  static constexpr int QSTRIDE = (QPLANE * 8 + 127) / 128 * 16;  // doubles
  static constexpr int FSTRIDE = (FPLANE * 8 + 127) / 128 * 16;
  static constexpr uint32_t BYTES = 8u * (2 * QPLANE + 2 * FPLANE);  // landed per tile
  static constexpr int BUF = 2 * QSTRIDE + 2 * FSTRIDE;             // doubles per buffer
  static constexpr size_t SMEM = 8u * 2 * BUF;                        // two buffers
};

// Tensor maps of a 2D FP64 master: q0, q1 (box QX x QY), f0, f1 (box TX x TY),
// in M.tmaps.  The twin's precision TW is read per tile.  Two tile buffers:
// the copies of a CTA's next tile land while it computes the current one.
template <int D>
__global__ void __launch_bounds__(BLOCK_THREADS, 8)
    kb_defect_tma(const DevPatch* __restrict__ PT, const Item* __restrict__ items,
                  const int* __restrict__ count, double* __restrict__ partials, int newstep_only,
                  int* __restrict__ err, TileRuns R) {
  static_assert(D == 2, "2D masters only");
  using F = Defect2;
  extern __shared__ __align__(1024) unsigned char def_raw[];
  __shared__ __align__(8) uint64_t bar[2];
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int n = *count;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  auto plane = [&](int buf, int k) {
    double* base = reinterpret_cast<double*>(def_raw) + buf * F::BUF;
    return k < 2 ? base + k * F::QSTRIDE : base + 2 * F::QSTRIDE + (k - 2) * F::FSTRIDE;
  };
  // Whether a patch takes part, remembered for the last patch asked about:
  // the tiles of a run mostly share their patch, so its record is read once
  // per patch rather than once per tile (each read is a round trip to L2).
  int part_patch = -1;
  bool part_ok = false;
  auto takes_part = [&](int p) {
    if (p != part_patch) {
      const DevPatch& M = PT[p];
      part_ok = M.active && !(newstep_only && !M.newstep);
      part_patch = p;
    }
    return part_ok;
  };
  // The CTA's next tile at or after list position `from` that takes part.
  auto next_tile = [&](int from) {
    for (int x = from; x < n; x = R.next(x))
      if (takes_part(items[x].patch)) return x;
    return n;
  };
  // Thread 0: the bulk copies of tile x into buffer buf.
  auto issue = [&](int x, int buf) {
    const Item it = items[x];
    const DevPatch& M = PT[it.patch];
    const CUtensorMapOpaque* maps = static_cast<const CUtensorMapOpaque*>(M.tmaps);
    const int lead = 128 / (int)sizeof(double) - 1;
    const int i0 = it.tx * F::TX + 1, j0 = it.ty * F::TY + 1;
    fence_proxy_async_smem();  // earlier generic reads of the buffer come first
    mbar_arrive_expect_tx(&bar[buf], F::BYTES);
    tma_load_2d(plane(buf, 0), &maps[0], lead + i0 - 2, j0 - 1, &bar[buf]);
    tma_load_2d(plane(buf, 1), &maps[1], lead + i0 - 2, j0 - 1, &bar[buf]);
    tma_load_2d(plane(buf, 2), &maps[2], lead + i0, j0, &bar[buf]);
    tma_load_2d(plane(buf, 3), &maps[3], lead + i0, j0, &bar[buf]);
  };
  uint32_t phase[2] = {0u, 0u};
  int mw_patch = -1;
  DevPatch M, W;
  int cur = next_tile(R.first()), buf = 0;
  if (cur < n && tid == 0) issue(cur, 0);
  while (cur < n) {
    // Buffer buf ^ 1 was last read by the previous tile, which ended with a
    // barrier (block_sum).
    const int nxt = next_tile(R.next(cur));
    if (nxt < n && tid == 0) issue(nxt, buf ^ 1);
    bool ok = true;
    if (tid == 0) ok = mbar_wait_backoff(&bar[buf], phase[buf], kWaitPolls);
    ok = __syncthreads_and(ok);
    if (ok && tid != 0) (void)mbar_try_wait(&bar[buf], phase[buf]);
    phase[buf] ^= 1u;
    if (!ok) {
      if (tid == 0) {
        atomicExch(err, kErrTmaTimeout);
        // Let the copies of the prefetched tile land before the CTA exits.
        if (nxt < n) (void)mbar_wait_backoff(&bar[buf ^ 1], phase[buf ^ 1], kWaitPolls);
      }
      break;
    }
    const double* sq0 = plane(buf, 0);
    const double* sq1 = plane(buf, 1);
    const double* sf0 = plane(buf, 2);
    const double* sf1 = plane(buf, 3);
    const Item it = items[cur];
    // The master and its twin, read again only when the patch changes.
    if (it.patch != mw_patch) {
      M = PT[it.patch];
      W = PT[M.twin];
      mw_patch = it.patch;
    }
    const int i0 = it.tx * F::TX + 1, j0 = it.ty * F::TY + 1;
    // defect_item's cells of this thread, from the staged tile.
    const int j = j0 + threadIdx.y;
    const int ic0 = (it.tx * 32 + threadIdx.x) * 2 + 1;
    double acc = 0.0;
    if (j <= M.n[1]) {
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const int i = ic0 + t;
        if (i > M.n[0]) break;
        const int sq = (i - (i0 - 2)) + (j - (j0 - 1)) * F::QX;
        const int sf = (i - i0) + (j - j0) * F::TX;
        Problem::Stencil<double, 2> s;
        s.pc = sq0[sq];
        s.mc = sq1[sq];
        s.pm[0] = sq0[sq - 1];
        s.pp[0] = sq0[sq + 1];
        s.mm[0] = sq1[sq - 1];
        s.mp[0] = sq1[sq + 1];
        s.pm[1] = sq0[sq - F::QX];
        s.pp[1] = sq0[sq + F::QX];
        s.mm[1] = sq1[sq - F::QX];
        s.mp[1] = sq1[sq + F::QX];
        double o0, o1;
        Problem::OperatorCell<double, 2>(s, M.tmp1, M.tmp2, M.alpha, o0, o1);
        const double r0 = sf0[sf] - o0, r1 = sf1[sf] - o1;
        acc += r0 * r0 + r1 * r1;
        const int64_t cw = cidx(W, i, j, 0);
        if (W.prec == PREC_F32) {
          fld<float>(W.f[0])[cw] = float(r0);
          fld<float>(W.f[1])[cw] = float(r1);
          fld<float>(W.bs)[cw] = float(s.pc);
          // A fused twin's pre-smoothing starts from a zero correction
          // without reading it (kb_smooth2), so only the others store it.
          if (!W.fused) {
            float* e0 = fld<float>(W.q[0]);
            float* e1 = fld<float>(W.q[1]);
            e0[cw] = 0.f;
            e1[cw] = 0.f;
            if (W.wt && near_boundary(W, i, j, 0, 2))
              write_through<float, 2>(W, e0, e1, i, j, 0, 0.f, 0.f);
          }
        } else {
          double* e0 = fld<double>(W.q[0]);
          double* e1 = fld<double>(W.q[1]);
          fld<double>(W.f[0])[cw] = r0;
          fld<double>(W.f[1])[cw] = r1;
          fld<double>(W.bs)[cw] = s.pc;
          e0[cw] = 0.0;
          e1[cw] = 0.0;
          if (W.wt && near_boundary(W, i, j, 0, 2))
            write_through<double, 2>(W, e0, e1, i, j, 0, 0.0, 0.0);
        }
      }
    }
    const double bsum = block_sum(acc);  // ends with a barrier: the buffer is free
    if (!newstep_only && tid == 0) partials[cur] = bsum;
    cur = nxt;
    buf ^= 1;
  }
}

}  // namespace bsam
