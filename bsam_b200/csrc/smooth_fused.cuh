// smooth_fused.cuh -- one launch per smoothing stage (LevelRelax, afas:523-547).
//
// The reference relaxes a level with nu red-black sweeps, i.e. 2*nu colour
// passes, each followed by SetGhost (afas:536-545).  Run as separate launches
// every pass reads the whole level from memory.  This kernel runs all four
// passes of a nu = 2 stage in one launch by temporal blocking:
//
//  * A CTA owns an in-plane tile of TX x TY interior cells (x, y) and streams
//    along z through a chunk of planes.  Planes of phi and mu are staged in a
//    shared-memory ring of NS slots by the TMA engine (cp.async.bulk, one bulk
//    copy per row of the 4-cell halo'd tile, completion on one mbarrier per
//    slot), PREFETCH planes ahead of use; f is read through L2.
//  * At stream step t, pass p (p = 1..4) updates plane t - 2p + 1 over the
//    tile grown by 4 - p cells in x and y.  Pass p on plane z only needs pass
//    p-1 on planes z-1..z+1 and within one cell, so the result is
//    bit-identical to running the passes one after another over the whole
//    level.  Halo cells are recomputed by each CTA that needs them (same
//    inputs, same result).
//  * Chunks in z overlap by the same wavefront: a chunk [zc0, zc1) loads
//    planes zc0-4 .. zc1+3, recomputing the planes its neighbour chunk owns.
//  * Neighbours across a physical face are read through the SetBC rule
//    (ghost = face map of the mirrored cell), so ghost cells are never staged;
//    the final values and their ghosts are written to the output buffer.
//
// Input and output are different buffers (q -> qb for pre-smoothing,
// qb -> q for post-smoothing) because neighbouring CTAs read each other's
// tiles as halo while the stage runs.
#pragma once
#include "kernels.cuh"

namespace bsam {

// ---- TMA / mbarrier helpers (sm_90+ PTX) -----------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return done != 0;
}
// Bulk global -> shared copy on the TMA engine (no multicast).  Both
// addresses 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Tiled 3D tensor copy global -> shared on the TMA engine (no multicast).
// The x coordinate times the element size is a multiple of 16 bytes at every
// call site (tile origins are multiples of 32 cells, see k_smooth3_fused).
__device__ __forceinline__ void tma_load_3d(void* dst, const void* tmap, int x, int y, int z,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, "
      "{%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Bounded wait on an mbarrier phase.  Returns false after `limit` polls; the
// caller records the failure and leaves without touching the stage's data.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* b, uint32_t parity, uint32_t limit) {
  for (uint32_t it = 0; it < limit; ++it) {
    if (mbar_try_wait(b, parity)) return true;
    if (it > 64) __nanosleep(64);
  }
  return false;
}

// Device-side view of a CUtensorMap (128 bytes, 64-byte aligned), built on
// the host with cuTensorMapEncodeTiled.
struct alignas(64) CUtensorMapOpaque {
  unsigned long long v[16];
};

constexpr uint32_t kWaitPolls = 1u << 22;   // about 0.3 s of polling
constexpr int kErrTmaTimeout = 1;

// ---- 3D fused stage ---------------------------------------------------------
//
// Staggered wavefront: at stream step t, pass p (p = 1..4) runs on plane
// z = t - 2p + 1.  With a lag of two planes per pass, the four passes of one
// step touch disjoint data: pass p reads the other colour on planes z-1..z+1,
// which pass p-1 finished in earlier steps and pass p+1 reaches only in later
// steps.  So the four passes of a step run concurrently between two barriers.
template <class T>
struct Fused3 {
  // Staged fields: phi, mu, f1, f2 and, for FP32 correction-form levels, the
  // base phi.  FP64 tiles are half as tall so that the ring fits in 227 KB.
  static constexpr int NFIELD = sizeof(T) == 4 ? 5 : 4;
  static constexpr int TX = 32, TY = sizeof(T) == 4 ? 16 : 8, H = 4;
  static constexpr int HX = TX + 2 * H, HY = TY + 2 * H;
  static constexpr int LAG = 2;                             // planes between passes
  static constexpr int PREFETCH = sizeof(T) == 4 ? 2 : 1;   // planes loaded ahead
  static constexpr int NS = 2 * 4 + 1 + PREFETCH;           // planes t-8 .. t+PREFETCH
  static constexpr int THREADS = 512;
  static constexpr int PLANE = HX * HY;
  static constexpr size_t SMEM = (size_t)NFIELD * NS * PLANE * sizeof(T) + NS * sizeof(uint64_t);
  static_assert((HX * sizeof(T)) % 16 == 0, "bulk rows must be multiples of 16 bytes");
  static_assert(SMEM <= 227 * 1024, "the stage ring must fit in one CTA's shared memory");
};

template <class T>
__device__ __forceinline__ T nb_or_face(bool at_face, int code, T self, const T* p, int off) {
  return at_face ? bc_map<T>(code, self) : p[off];
}

// Relax one cell (i, j, z) of the staged tile: RelaxGrid3D's update
// (problem.f90:489-513), neighbours across physical faces by the SetBC rule.
// so/som/sop: slot offsets of planes z, z-1, z+1; zl/zh: z on a z face.
template <class T>
__device__ __forceinline__ void fused3_cell(const DevPatch& P, T* sphi, T* smu, const T* sf0,
                                            const T* sf1, const T* sbs, int lc, int so, int som,
                                            int sop, bool xl, bool xh, bool yl, bool yh, bool zl,
                                            bool zh) {
  using C = Fused3<T>;
  const T f0 = sf0[so + lc], f1 = sf1[so + lc];
  const T* ph = sphi + lc;
  const T* mu_ = smu + lc;
  Problem::Stencil<T, 3> s;
  s.pc = ph[so];
  s.mc = mu_[so];
  if (!(xl | xh | yl | yh | zl | zh)) {
    s.pm[0] = ph[so - 1];
    s.pp[0] = ph[so + 1];
    s.pm[1] = ph[so - C::HX];
    s.pp[1] = ph[so + C::HX];
    s.pm[2] = ph[som];
    s.pp[2] = ph[sop];
    s.mm[0] = mu_[so - 1];
    s.mp[0] = mu_[so + 1];
    s.mm[1] = mu_[so - C::HX];
    s.mp[1] = mu_[so + C::HX];
    s.mm[2] = mu_[som];
    s.mp[2] = mu_[sop];
  } else {
    s.pm[0] = nb_or_face(xl, P.bc[0], s.pc, ph, so - 1);
    s.pp[0] = nb_or_face(xh, P.bc[1], s.pc, ph, so + 1);
    s.pm[1] = nb_or_face(yl, P.bc[2], s.pc, ph, so - C::HX);
    s.pp[1] = nb_or_face(yh, P.bc[3], s.pc, ph, so + C::HX);
    s.pm[2] = nb_or_face(zl, P.bc[4], s.pc, ph, som);
    s.pp[2] = nb_or_face(zh, P.bc[5], s.pc, ph, sop);
    s.mm[0] = nb_or_face(xl, P.bc[0], s.mc, mu_, so - 1);
    s.mp[0] = nb_or_face(xh, P.bc[1], s.mc, mu_, so + 1);
    s.mm[1] = nb_or_face(yl, P.bc[2], s.mc, mu_, so - C::HX);
    s.mp[1] = nb_or_face(yh, P.bc[3], s.mc, mu_, so + C::HX);
    s.mm[2] = nb_or_face(zl, P.bc[4], s.mc, mu_, som);
    s.mp[2] = nb_or_face(zh, P.bc[5], s.mc, mu_, sop);
  }
  T phi, mu;
  if (C::NFIELD == 5 && P.delta)
    Problem::RelaxCell<T, 3, true>(s, f0, f1, T(P.tmp1), T(P.tmp2), T(P.tmp3), T(P.alpha), phi,
                                   mu, sbs[so + lc]);
  else
    Problem::RelaxCell<T, 3>(s, f0, f1, T(P.tmp1), T(P.tmp2), T(P.tmp3), T(P.alpha), phi, mu);
  sphi[so + lc] = phi;
  smu[so + lc] = mu;
}

// dir = 0: q -> qb (pre-smoothing); dir = 1: qb -> q (post-smoothing).
// color0 = colour of the first pass (0: even i+j+k, the reference's ipass 1).
template <class T>
__global__ void __launch_bounds__(Fused3<T>::THREADS, 1)
    k_smooth3_fused(const DevPatch* __restrict__ PT, const Item* __restrict__ items, int dir,
                    int color0, int* __restrict__ err) {
  using C = Fused3<T>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  T* sphi = reinterpret_cast<T*>(smem_raw);
  T* smu = sphi + C::NS * C::PLANE;
  T* sf0 = smu + C::NS * C::PLANE;
  T* sf1 = sf0 + C::NS * C::PLANE;
  T* sbs = sf1 + C::NS * C::PLANE;  // only when NFIELD == 5
  uint64_t* bar = reinterpret_cast<uint64_t*>(sphi + C::NFIELD * C::NS * C::PLANE);

  const Item it = items[blockIdx.x];
  const DevPatch P = PT[it.patch];  // by value: fields stay in registers
  const int n0 = P.n[0], n1 = P.n[1], n2 = P.n[2];
  const int x0 = it.tx * C::TX, y0 = it.ty * C::TY;
  const int zc0 = it.tz * P.zchunk + 1;
  const int zc1 = min(zc0 + P.zchunk, n2 + 1);
  T* out0 = fld<T>(dir ? P.q[0] : P.qb[0]);
  T* out1 = fld<T>(dir ? P.q[1] : P.qb[1]);

  if (threadIdx.x < C::NS) mbar_init(&bar[threadIdx.x], 1);
  fence_mbar_init();
  __syncthreads();

  // Only interior cells of the staged boxes are ever read (a neighbour across
  // a physical face comes from the SetBC rule instead).
  const int nfield = (C::NFIELD == 5 && P.delta) ? 5 : 4;
  const uint32_t box_bytes = (uint32_t)(nfield * C::PLANE * sizeof(T));
  const int lead = 128 / (int)sizeof(T) - 1;

  // Issues the bulk copies of plane z (same decision in every thread; warp 0
  // issues).  Returns true when a copy was issued.
  // One tiled TMA box (HX x HY x 1) per field per plane.  The maps address
  // each field from its allocation start, whose first element sits `lead`
  // elements before element (0,0,0); boxes reaching outside the array are
  // zero-filled by the TMA unit (those cells are never read).
  auto issue = [&](int z) -> bool {
    if (z < 1 || z > n2) return false;
    if (threadIdx.x == 0) {
      const int s = z % C::NS;
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&bar[s], box_bytes);
      const CUtensorMapOpaque* maps = static_cast<const CUtensorMapOpaque*>(P.tmaps);
      const int x = x0 - 3 + lead;
      for (int fidx = 0; fidx < nfield; ++fidx) {
        const int m = fidx < 2 ? fidx + 2 * dir : fidx + 2;  // q0 q1 | qb0 qb1 | f0 f1 bs
        tma_load_3d(sphi + (fidx * C::NS + s) * C::PLANE, &maps[m], x, y0 - 3, z, &bar[s]);
      }
    }
    return true;
  };

  // Pass p covers planes [zc0 - (4-p), zc1 - 1 + (4-p)]: loads [zc0-4, zc1+3].
  const int ts = zc0 - 4, te = zc1 - 1 + 2 * 4 - 1 + 1;  // last step stores plane zc1-1
  uint32_t phase = 0, pending = 0;
  for (int z = ts; z <= ts + C::PREFETCH - 1; ++z)
    if (z <= zc1 + 3 && issue(z)) pending |= 1u << (z % C::NS);
  bool ok = true;
  // Region widths per pass (tile grown by 4 - p) and the per-step item count.
  constexpr int M = C::HX / 2;
  for (int t = ts; t <= te; ++t) {
    const int zn = t + C::PREFETCH;
    if (zn <= zc1 + 3 && issue(zn)) pending |= 1u << (zn % C::NS);
    if (t >= 1 && t <= n2 && t <= zc1 + 3) {
      const int s = t % C::NS;
      const bool got = mbar_wait_bounded(&bar[s], (phase >> s) & 1u, kWaitPolls);
      if (__syncthreads_or(!got)) {
        ok = false;
        break;
      }
      phase ^= 1u << s;
      pending &= ~(1u << s);
    }
    // The four passes of this step, as one flat list of cell slots.
    int za[4], ia[4], ib[4], ja[4], rows[4], base[4], col[4];
    int total = 0;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const int g = 3 - p, z = t - 2 * p - 1;
      za[p] = z;
      col[p] = (p & 1) ? 1 - color0 : color0;
      ia[p] = max(1, x0 + 1 - g);
      ib[p] = min(n0, x0 + C::TX + g);
      ja[p] = max(1, y0 + 1 - g);
      const int jb = min(n1, y0 + C::TY + g);
      const bool on = z >= 1 && z <= n2 && z >= zc0 - g && z <= zc1 - 1 + g && ia[p] <= ib[p] &&
                      ja[p] <= jb;
      rows[p] = on ? jb - ja[p] + 1 : 0;
      base[p] = total;
      total += rows[p] * M;
    }
    for (int idx = threadIdx.x; idx < total; idx += C::THREADS) {
      // Select this slot's pass with constant indices only (keeps the
      // per-pass parameters in registers).
      int z = za[0], a = ia[0], b = ib[0], j0 = ja[0], c = col[0], loc = idx;
#pragma unroll
      for (int q = 1; q < 4; ++q)
        if (idx >= base[q]) {
          z = za[q];
          a = ia[q];
          b = ib[q];
          j0 = ja[q];
          c = col[q];
          loc = idx - base[q];
        }
      const int r = loc / M, m = loc - r * M;
      const int j = j0 + r;
      const int i = a + ((a + j + z + c) & 1) + 2 * m;
      if (i <= b) {
        const int so = (z % C::NS) * C::PLANE;
        const int som = ((z + C::NS - 1) % C::NS) * C::PLANE;
        const int sop = ((z + 1) % C::NS) * C::PLANE;
        const int lc = (j - (y0 - 3)) * C::HX + (i - (x0 - 3));
        fused3_cell<T>(P, sphi, smu, sf0, sf1, sbs, lc, so, som, sop, i == 1, i == n0, j == 1,
                       j == n1, z == 1, z == n2);
      }
    }
    // Store plane t - 8, finished by pass 4 in the previous step.
    const int zs = t - 8;
    if (zs >= zc0 && zs < zc1) {
      const int sz = (zs % C::NS) * C::PLANE;
      for (int idx = threadIdx.x; idx < C::TX * C::TY; idx += C::THREADS) {
        const int j = y0 + 1 + idx / C::TX, i = x0 + 1 + idx % C::TX;
        if (i > n0 || j > n1) continue;
        const int lc = (j - (y0 - 3)) * C::HX + (i - (x0 - 3));
        const T a = sphi[sz + lc], b = smu[sz + lc];
        const int64_t c = cidx(P, i, j, zs);
        out0[c] = a;
        out1[c] = b;
        if (near_boundary(P, i, j, zs, 3)) write_through<T, 3>(P, out0, out1, i, j, zs, a, b);
      }
    }
    __syncthreads();
  }
  if (!ok) {
    if (threadIdx.x == 0) atomicExch(err, kErrTmaTimeout);
    // Drain: wait (bounded) for the copies this CTA still has in flight.
    for (int s = 0; s < C::NS; ++s)
      if (pending & (1u << s)) mbar_wait_bounded(&bar[s], (phase >> s) & 1u, kWaitPolls);
  }
}

}  // namespace bsam
