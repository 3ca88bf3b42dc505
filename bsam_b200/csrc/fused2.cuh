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
// Thread layout of a pass: warp w takes a contiguous band of row pairs, lane
// l the columns 2l, 2l+1 of its rows (smooth_band).  TX = 56 keeps the widest
// pass (TX + 6 cells) within the 64 columns of a warp.
#pragma once
#include <type_traits>

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

// Physical face ghosts of a shared tile, refreshed from the interior cells
// next to them: ghost = the face map of SetBC2D (boundary.f90:661-738) of its
// mirror cell.  In a 5-point colour pass a face ghost is read only by its own
// mirror cell, the one that writes it through in the reference's order
// (SetGhost after the pass), so refreshing every face ghost of the tile after
// a pass gives the ghosts the next pass reads exactly; corners are never
// read.  Only tiles that hold a patch face call this.
template <class T>
__device__ __forceinline__ void refresh_faces(const DevPatch& P, T* s0, T* s1, int gx0, int gy0) {
  constexpr int RX = Fused2<T>::RX, RY = Fused2<T>::RY;
  const int n0 = P.n[0], n1 = P.n[1];
  // Interior cells held by the tile with both neighbours in the tile.
  const int cx0 = max(1, 1 - gx0), cx1 = min(RX - 1, n0 + 1 - gx0);
  const int cy0 = max(1, 1 - gy0), cy1 = min(RY - 1, n1 + 1 - gy0);
  const int t = threadIdx.x;
  if (t < RY) {
    const int sy = t;
    if (sy >= cy0 && sy < cy1) {
      const int lo = 1 - gx0, hi = n0 - gx0;
      if (P.bc[0] != BC_NONE && lo >= 1 && lo <= RX - 2) {
        const int c = sy * RX + lo;
        s0[c - 1] = bc_map<T>(P.bc[0], s0[c]);
        s1[c - 1] = bc_map<T>(P.bc[0], s1[c]);
      }
      if (P.bc[1] != BC_NONE && hi >= 1 && hi <= RX - 2) {
        const int c = sy * RX + hi;
        s0[c + 1] = bc_map<T>(P.bc[1], s0[c]);
        s1[c + 1] = bc_map<T>(P.bc[1], s1[c]);
      }
    }
  } else if (t >= 64 && t < 64 + RX) {
    const int sx = t - 64;
    if (sx >= cx0 && sx < cx1) {
      const int lo = 1 - gy0, hi = n1 - gy0;
      if (P.bc[2] != BC_NONE && lo >= 1 && lo <= RY - 2) {
        const int c = lo * RX + sx;
        s0[c - RX] = bc_map<T>(P.bc[2], s0[c]);
        s1[c - RX] = bc_map<T>(P.bc[2], s1[c]);
      }
      if (P.bc[3] != BC_NONE && hi >= 1 && hi <= RY - 2) {
        const int c = hi * RX + sx;
        s0[c + RX] = bc_map<T>(P.bc[3], s0[c]);
        s1[c + RX] = bc_map<T>(P.bc[3], s1[c]);
      }
    }
  }
}

template <class T> struct Pair2;
template <> struct Pair2<float> { using V = float2; };
template <> struct Pair2<double> { using V = double2; };

// Constants of a level's FP32 Newton update as packed pairs, with the signs
// folded in (negation is exact, so -x * y, x * -y and -(x * y) round alike).
struct RelaxK2 {
  float2 tmp1, ntmp2, tmp3, alpha, nalpha, three, mhalf, one, a12, na12;
};

__device__ __forceinline__ float2 splat2(float a) { return make_float2(a, a); }

__device__ __forceinline__ RelaxK2 relax_k2(float tmp1, float tmp2, float tmp3, float alpha) {
  RelaxK2 K;
  K.tmp1 = splat2(tmp1);
  K.ntmp2 = splat2(-tmp2);
  K.tmp3 = splat2(tmp3);
  K.alpha = splat2(alpha);
  K.nalpha = splat2(-alpha);
  K.three = splat2(3.f);
  K.mhalf = splat2(-0.5f);
  K.one = splat2(1.f);
  // a12 = tmp1 * (m1 + m2 + m3 + m4) with Mob = 1: tmp1 * 4, exact.
  K.a12 = splat2(tmp1 * 4.f);
  K.na12 = splat2(-(tmp1 * 4.f));
  return K;
}

// Paired FP32 operations (PTX add/mul/fma .rn.f32x2, Blackwell), each half
// rounded to nearest; written out as PTX so that every one stays a separately
// rounded operation.
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
  float2 d;
  asm("{.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
  float2 d;
  asm("{.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
  float2 d;
  asm("{.reg .b64 ra, rb, rc, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "mov.b64 rc, {%6, %7};\n\tfma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
}

// RelaxCell's FP32 Newton update (problem_ch.cuh) of two cells at once, one
// in each half of the packed pairs, with Blackwell's paired FP32 arithmetic.
// Every operation is RelaxCell's, in its order and rounding (x - 0.5 is
// x + (-0.5); the negated products are the same products of negated
// operands), so each half equals RelaxCell<float, 2> bit for bit.  The
// correction form's terms (cfull and DfcDelta) are taken one half at a time
// with scalar operations: evaluated paired, the sum of the polynomial's terms
// differed in its last bit from the scalar sum in about 1 of 10^4 cases in a
// probe of random stencils, which the scalar form does not.
template <bool DELTA>
__device__ __forceinline__ void relax_pair_f32(float2 pc, float2 pw, float2 pe, float2 ps,
                                               float2 pn, float2 mw, float2 me, float2 ms,
                                               float2 mn, float2 f0, float2 f1, float2 bs,
                                               const RelaxK2& K, float2& phi, float2& mu) {
  const float2 smu = add2(add2(add2(mw, me), ms), mn);
  const float2 sph = add2(add2(add2(pe, pw), pn), ps);
  float2 cmh, nl;
  if (DELTA) {
    // cfull - 1/2 with cfull = base + e, and DfcDelta(base, e) = alpha e
    // (3 c^2 + 3 c e + e^2), c = base - 1/2: RelaxCell's scalar operations.
    auto half = [&](float b, float e, float& cm, float& n) {
      cm = __fadd_rn(__fadd_rn(b, e), -0.5f);
      const float c = __fadd_rn(b, -0.5f);
      const float c3 = __fmul_rn(3.f, c);
      const float poly =
          __fadd_rn(__fadd_rn(__fmul_rn(c3, c), __fmul_rn(c3, e)), __fmul_rn(e, e));
      n = __fmul_rn(__fmul_rn(K.alpha.x, e), poly);
    };
    half(bs.x, pc.x, cmh.x, nl.x);
    half(bs.y, pc.y, cmh.y, nl.y);
  } else {
    cmh = add2(pc, K.mhalf);
    nl = mul2(mul2(mul2(cmh, cmh), cmh), K.alpha);  // Dfc
  }
  const float2 u = mul2(mul2(K.three, cmh), cmh);
  const float2 d2 = mul2(u, K.alpha);     // D2fc(cfull)
  const float2 nd2 = mul2(u, K.nalpha);   // -D2fc(cfull)
  const float2 na21 = add2(d2, K.tmp3);   // -a21
  const float2 b1 = fma2(K.tmp1, smu, f0);
  const float2 b2 = fma2(K.ntmp2, sph, fma2(nd2, pc, add2(f1, nl)));
  const float2 det = fma2(K.a12, na21, K.one);
  const float2 r = make_float2(rcp_approx(det.x), rcp_approx(det.y));
  phi = mul2(fma2(K.na12, b2, b1), r);
  mu = mul2(fma2(na21, b1, b2), r);
}

// The Newton updates of cells A (row y) and B (row y + 1), by the working
// type: FP32 as a packed pair, FP64 one cell at a time in the reference's
// operation order.  Stencil order of a/b: pc, pw, pe, ps, pn, mw, me, ms, mn,
// f0, f1, base.
// The FP32 pair with the Cahn-Hilliard Newton step in paired arithmetic.
template <bool DELTA> struct RelaxPairF32 {
  RelaxK2 K;
  __device__ __forceinline__ explicit RelaxPairF32(const DevPatch& P)
      : K(relax_k2(float(P.tmp1), float(P.tmp2), float(P.tmp3), float(P.alpha))) {}
  __device__ __forceinline__ void operator()(const float (&a)[12], const float (&b)[12],
                                             float& pa, float& ma, float& pb, float& mb) const {
    float2 phi, mu;
    auto v = [&](int k) { return make_float2(a[k], b[k]); };
    relax_pair_f32<DELTA>(v(0), v(1), v(2), v(3), v(4), v(5), v(6), v(7), v(8), v(9), v(10),
                          v(11), K, phi, mu);
    pa = phi.x;
    pb = phi.y;
    ma = mu.x;
    mb = mu.y;
  }
};
// Any pair cell by cell through the problem module's RelaxCell.
template <class T, bool DELTA> struct RelaxPairScalar {
  T tmp1, tmp2, tmp3, alpha;
  __device__ __forceinline__ explicit RelaxPairScalar(const DevPatch& P)
      : tmp1(T(P.tmp1)), tmp2(T(P.tmp2)), tmp3(T(P.tmp3)), alpha(T(P.alpha)) {}
  __device__ __forceinline__ void one(const T (&a)[12], T& p, T& m) const {
    Problem::Stencil<T, 2> st;
    st.pc = a[0];
    st.pm[0] = a[1];
    st.pp[0] = a[2];
    st.pm[1] = a[3];
    st.pp[1] = a[4];
    st.mm[0] = a[5];
    st.mp[0] = a[6];
    st.mm[1] = a[7];
    st.mp[1] = a[8];
    st.mc = T(0);  // the Newton update does not read mu at the cell
    if constexpr (DELTA)
      Problem::RelaxCell<T, 2, true>(st, a[9], a[10], tmp1, tmp2, tmp3, alpha, p, m, a[11]);
    else
      Problem::RelaxCell<T, 2>(st, a[9], a[10], tmp1, tmp2, tmp3, alpha, p, m);
  }
  __device__ __forceinline__ void operator()(const T (&a)[12], const T (&b)[12], T& pa, T& ma,
                                             T& pb, T& mb) const {
    one(a, pa, ma);
    one(b, pb, mb);
  }
};

// The pair form of a level: paired FP32 arithmetic where the problem module
// allows it (its Newton step is the one relax_pair_f32 evaluates), else cell
// by cell.
template <class T, bool DELTA>
using RelaxPair =
    typename std::conditional<std::is_same<T, float>::value && Problem::paired_f32,
                              RelaxPairF32<DELTA>, RelaxPairScalar<T, DELTA>>::type;

// One colour pass over a band of row pairs of the shared tile.  Lane l holds
// columns 2l and 2l+1 of every row it touches, read as one vector: per row
// pair (y, y+1) it updates cell A = (2l + PA, y) and cell B = (2l + 1 - PA,
// y + 1), the pass's colour in both rows (PA, the column parity of the
// colour in row y, is the same for every pair of a pass).  The four
// neighbours of A and B are the other colour, which the pass does not write:
// the rows above and below come from the vectors of rows y - 1 .. y + 2
// (rows y + 1 and y + 2 carry over to the next pair as its y - 1 and y), the
// column beyond the lane's pair from the neighbouring lane by a shuffle.
// Columns outside [xa, xb) and row yb are computed but not stored (at the
// tile's outermost columns the shuffled neighbour is the lane's own value).
template <class T, bool DELTA, int PA>
__device__ __forceinline__ void smooth_band(T* s0, T* s1, const T* sf0, const T* sf1,
                                            const T* sbs, int ylo, int yhi, int yb, int xa,
                                            int xb, int lane, const RelaxPair<T, DELTA>& R) {
  using V = typename Pair2<T>::V;
  constexpr int RX = Fused2<T>::RX;
  constexpr int RV = RX / 2;  // vectors per shared row
  const V* v0 = reinterpret_cast<const V*>(s0) + lane;
  const V* v1 = reinterpret_cast<const V*>(s1) + lane;
  const V* vf0 = reinterpret_cast<const V*>(sf0) + lane;
  const V* vf1 = reinterpret_cast<const V*>(sf1) + lane;
  const V* vbs = reinterpret_cast<const V*>(sbs) + lane;
  const int xA = 2 * lane + PA, xB = 2 * lane + 1 - PA;
  const bool inA = xA >= xa && xA < xb, inB = xB >= xa && xB < xb;
  constexpr unsigned FULL = 0xffffffffu;
  V ps = v0[(ylo - 1) * RV], p0 = v0[ylo * RV];
  V ms = v1[(ylo - 1) * RV], m0 = v1[ylo * RV];
#pragma unroll 2
  for (int y = ylo; y < yhi; y += 2) {
    const V p1 = v0[(y + 1) * RV], p2 = v0[(y + 2) * RV];
    const V m1 = v1[(y + 1) * RV], m2 = v1[(y + 2) * RV];
    const V fa0 = vf0[y * RV], fb0 = vf0[(y + 1) * RV];
    const V fa1 = vf1[y * RV], fb1 = vf1[(y + 1) * RV];
    V ba{}, bb{};
    if constexpr (DELTA) {
      ba = vbs[y * RV];
      bb = vbs[(y + 1) * RV];
    }
    T a[12], b[12];
    if (PA == 0) {
      // A = column 2l of row y, B = column 2l + 1 of row y + 1.
      const T pwA = __shfl_up_sync(FULL, p0.y, 1), mwA = __shfl_up_sync(FULL, m0.y, 1);
      const T peB = __shfl_down_sync(FULL, p1.x, 1), meB = __shfl_down_sync(FULL, m1.x, 1);
      a[0] = p0.x; a[1] = pwA; a[2] = p0.y; a[3] = ps.x; a[4] = p1.x;
      a[5] = mwA; a[6] = m0.y; a[7] = ms.x; a[8] = m1.x;
      a[9] = fa0.x; a[10] = fa1.x; a[11] = ba.x;
      b[0] = p1.y; b[1] = p1.x; b[2] = peB; b[3] = p0.y; b[4] = p2.y;
      b[5] = m1.x; b[6] = meB; b[7] = m0.y; b[8] = m2.y;
      b[9] = fb0.y; b[10] = fb1.y; b[11] = bb.y;
    } else {
      // A = column 2l + 1 of row y, B = column 2l of row y + 1.
      const T peA = __shfl_down_sync(FULL, p0.x, 1), meA = __shfl_down_sync(FULL, m0.x, 1);
      const T pwB = __shfl_up_sync(FULL, p1.y, 1), mwB = __shfl_up_sync(FULL, m1.y, 1);
      a[0] = p0.y; a[1] = p0.x; a[2] = peA; a[3] = ps.y; a[4] = p1.y;
      a[5] = m0.x; a[6] = meA; a[7] = ms.y; a[8] = m1.y;
      a[9] = fa0.y; a[10] = fa1.y; a[11] = ba.y;
      b[0] = p1.x; b[1] = pwB; b[2] = p1.y; b[3] = p0.x; b[4] = p2.x;
      b[5] = mwB; b[6] = m1.y; b[7] = m0.x; b[8] = m2.x;
      b[9] = fb0.x; b[10] = fb1.x; b[11] = bb.x;
    }
    T pA, mA, pB, mB;
    R(a, b, pA, mA, pB, mB);
    if (inA) {
      s0[y * RX + xA] = pA;
      s1[y * RX + xA] = mA;
    }
    if (inB && y + 1 < yb) {
      s0[(y + 1) * RX + xB] = pB;
      s1[(y + 1) * RX + xB] = mB;
    }
    ps = p1;
    p0 = p2;
    ms = m1;
    m0 = m2;
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
// MINB CTAs per SM (the shared tile allows four): four caps a thread at 64
// registers, three at 85.  NBUF = 2: two tile buffers per CTA (two CTAs per
// SM), the copies of the CTA's next tile land while it computes the current
// one.
template <class T, bool DELTA, int MINB = 4, int NBUF = 1>
__global__ void __launch_bounds__(Fused2<T>::THREADS, MINB)
    kb_smooth2(const DevPatch* __restrict__ PT, const Item* __restrict__ items,
               const int* __restrict__ count, int dir, int nu, int upd, int corr,
               int restr, int* __restrict__ err, TileRuns R) {
  using F = Fused2<T>;
  static_assert(NBUF == 1 || NBUF == 2, "one or two tile buffers");
  constexpr int NPL = DELTA ? 5 : 4;  // planes per buffer
  extern __shared__ __align__(1024) unsigned char smem2_raw[];
  __shared__ __align__(8) uint64_t bar[NBUF];
  auto plane = [&](int buf, int k) {
    return reinterpret_cast<T*>(smem2_raw) + (size_t)(buf * NPL + k) * F::PLANE;
  };
  const int n = *count;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int npass = 2 * nu;
  if (tid == 0) {
    for (int k = 0; k < NBUF; ++k) mbar_init(&bar[k], 1);
    fence_mbar_init();
  }
  __syncthreads();
  // The correction of the mixed form's finest working level is zero at the
  // start of every V-cycle (the defect starts a new correction): its
  // pre-smoothing stage fills the state planes with zeros instead of reading
  // them (the defect does not store them either).
  auto zero_start_of = [&](const DevPatch& P) { return DELTA && dir == 0 && P.master >= 0; };
  // The CTA's next tile at or after list position `from` whose patch runs.
  auto next_tile = [&](int from) {
    for (int x = from; x < n; x = R.next(x))
      if (PT[items[x].patch].active) return x;
    return n;
  };
  // Thread 0: the tensor copies of tile x into buffer buf.
  auto issue = [&](int x, int buf) {
    const Item it = items[x];
    const DevPatch& P = PT[it.patch];
    const int gx0 = it.tx * F::TX + 1 - F::H, gy0 = it.ty * F::TY + 1 - F::H;
    const int lead = 128 / (int)sizeof(T) - 1;
    const bool zs = zero_start_of(P);
    const CUtensorMapOpaque* maps = static_cast<const CUtensorMapOpaque*>(P.tmaps);
    const int m0 = dir == 0 ? 0 : 2;
    const uint32_t pl = (uint32_t)(sizeof(T) * F::PLANE);
    fence_proxy_async_smem();  // earlier generic accesses to the buffer come first
    mbar_arrive_expect_tx(&bar[buf], pl * (uint32_t)(NPL - (zs ? 2 : 0)));
    const int xc = gx0 + lead;  // column of element (gx0, *) from the allocation start
    if (!zs) {
      tma_load_2d(plane(buf, 0), &maps[m0], xc, gy0, &bar[buf]);
      tma_load_2d(plane(buf, 1), &maps[m0 + 1], xc, gy0, &bar[buf]);
    }
    tma_load_2d(plane(buf, 2), &maps[4], xc, gy0, &bar[buf]);
    tma_load_2d(plane(buf, 3), &maps[5], xc, gy0, &bar[buf]);
    if (DELTA) tma_load_2d(plane(buf, 4), &maps[6], xc, gy0, &bar[buf]);
  };
  uint32_t phase[NBUF];
  for (int k = 0; k < NBUF; ++k) phase[k] = 0u;
  int cur = next_tile(R.first()), buf = 0;
  if (cur < n && tid == 0) issue(cur, 0);
  while (cur < n) {
    const int nxt = next_tile(R.next(cur));
    // Two buffers: the next tile's copies go into the other one, last read
    // by the previous tile (which ended with a barrier).
    if (NBUF == 2 && nxt < n && tid == 0) issue(nxt, buf ^ 1);
    T* s0 = plane(buf, 0);
    T* s1 = plane(buf, 1);
    T* sf0 = plane(buf, 2);
    T* sf1 = plane(buf, 3);
    T* sbs = plane(buf, DELTA ? 4 : 3);
    const Item it = items[cur];
    const DevPatch P = PT[it.patch];
    const int gx0 = it.tx * F::TX + 1 - F::H;  // global i of shared column 0
    const int gy0 = it.ty * F::TY + 1 - F::H;  // global j of shared row 0
    if (zero_start_of(P))
      for (int c = tid; c < F::PLANE; c += F::THREADS) {
        s0[c] = T(0);
        s1[c] = T(0);
      }
    // One thread polls (with back-off, so that the waiting CTA takes no issue
    // slots from the CTAs computing beside it); after the barrier every
    // thread observes the completed phase itself.
    bool ok = true;
    if (tid == 0) ok = mbar_wait_backoff(&bar[buf], phase[buf], kWaitPolls);
    ok = __syncthreads_and(ok);
    if (ok && tid != 0) (void)mbar_try_wait(&bar[buf], phase[buf]);
    if (!ok) {
      // The launch's results are void (the host reports the error).  Before
      // the CTA exits, give the copies it started one more bounded wait each,
      // so that none is still writing into shared memory when the CTA ends.
      if (tid == 0) {
        atomicExch(err, kErrTmaTimeout);
        (void)mbar_wait_backoff(&bar[buf], phase[buf], kWaitPolls);
        if (NBUF == 2 && nxt < n)
          (void)mbar_wait_backoff(&bar[buf ^ 1], phase[buf ^ 1], kWaitPolls);
      }
      break;
    }
    phase[buf] ^= 1u;
    const int n0 = P.n[0], n1 = P.n[1];
    // A tile that holds a physical face of the patch refreshes the face
    // ghosts in shared memory after every change of its cells and writes
    // them through to HBM; the other tiles need neither (uniform per CTA).
    const bool edge_tile = P.wt && (gx0 <= 1 || gx0 + F::RX - 1 >= n0 || gy0 <= 1 ||
                                    gy0 + F::RY - 1 >= n1);
    if (corr && P.parent >= 0) {
      const DevPatch R = PT[P.parent];
      if (P.pprec == PREC_F32) correct_tile2<T, float>(P, R, s0, s1, gx0, gy0);
      else correct_tile2<T, double>(P, R, s0, s1, gx0, gy0);
      __syncthreads();
      if (edge_tile) {
        refresh_faces<T>(P, s0, s1, gx0, gy0);
        __syncthreads();
      }
    }
    T* o0 = fld<T>(dir == 0 ? P.qb[0] : P.q[0]);
    T* o1 = fld<T>(dir == 0 ? P.qb[1] : P.q[1]);
    const RelaxPair<T, DELTA> relax(P);
    for (int p = 0; p < npass; ++p) {
      const int color = p & 1;
      const int grow = npass - 1 - p;
      // Region of this pass in shared coordinates, clipped to the interior.
      const int xa = max(F::H - grow, 1 - gx0), xb = min(F::H + F::TX + grow, n0 + 1 - gx0);
      const int ya = max(F::H - grow, 1 - gy0), yb = min(F::H + F::TY + grow, n1 + 1 - gy0);
      // Row pairs from ya, split into contiguous bands, one per warp.
      const int npairs = (yb - ya + 1) >> 1;
      const int per = (npairs + F::WARPS - 1) / F::WARPS;
      const int k0 = warp * per, k1 = min(k0 + per, npairs);
      // Column parity of the pass's colour in the rows ya, ya + 2, ...:
      // (i + j) & 1 == color with i = gx0 + x, j = gy0 + y.
      const int pa = (gx0 + gy0 + ya + color) & 1;
      if (k0 < k1) {
        if (pa == 0)
          smooth_band<T, DELTA, 0>(s0, s1, sf0, sf1, sbs, ya + 2 * k0, ya + 2 * k1, yb, xa, xb,
                                   lane, relax);
        else
          smooth_band<T, DELTA, 1>(s0, s1, sf0, sf1, sbs, ya + 2 * k0, ya + 2 * k1, yb, xa, xb,
                                   lane, relax);
      }
      __syncthreads();
      if (edge_tile && p + 1 < npass) {
        refresh_faces<T>(P, s0, s1, gx0, gy0);
        __syncthreads();
      }
    }
    using V = typename Pair2<T>::V;
    // Columns 2l, 2l + 1 of the tile's interior: every pair starts at an odd
    // global column, so the pair is one aligned vector in shared memory, in
    // the level's rows and in the FP64 master's rows.
    const int lx = 2 * lane;
    const int gi = gx0 + F::H + lx;  // global column of the lane's first cell
    if (upd && P.master >= 0) {
      const DevPatch M = PT[P.master];
      double* m0 = fld<double>(M.q[0]);
      double* m1 = fld<double>(M.q[1]);
      if (lx < F::TX && gi <= n0)
        for (int ly = warp; ly < F::TY; ly += F::WARPS) {
          const int j = gy0 + F::H + ly;
          if (j > n1) break;
          const int srow = (F::H + ly) * F::RX + F::H;
          if (!edge_tile && gi + 1 <= n0) {
            const V e0 = *reinterpret_cast<const V*>(s0 + srow + lx);
            const V e1 = *reinterpret_cast<const V*>(s1 + srow + lx);
            double2* a0 = reinterpret_cast<double2*>(m0 + cidx(M, gi, j, 0));
            double2* a1 = reinterpret_cast<double2*>(m1 + cidx(M, gi, j, 0));
            double2 x0 = *a0, x1 = *a1;
            x0.x = x0.x + (double)e0.x;
            x0.y = x0.y + (double)e0.y;
            x1.x = x1.x + (double)e1.x;
            x1.y = x1.y + (double)e1.y;
            *a0 = x0;
            *a1 = x1;
            continue;
          }
          for (int d = 0; d < 2; ++d) {
            const int i = gi + d;
            if (i > n0) break;
            const int64_t c = cidx(M, i, j, 0);
            const double na = m0[c] + (double)s0[srow + lx + d];
            const double nb = m1[c] + (double)s1[srow + lx + d];
            m0[c] = na;
            m1[c] = nb;
            if (M.wt && near_boundary(M, i, j, 0, 2))
              write_through<double, 2>(M, m0, m1, i, j, 0, na, nb);
          }
        }
    } else {
      if (restr && P.parent >= 0) {
        const DevPatch R = PT[P.parent];
        if (P.pprec == PREC_F32) restrict_tile2<T, float, DELTA>(P, R, s0, s1, sbs, gx0, gy0);
        else restrict_tile2<T, double, DELTA>(P, R, s0, s1, sbs, gx0, gy0);
      }
      // Write back the tile's interior cells (warps over rows, lanes along
      // them, a pair per lane), ghosts by write-through on edge tiles.
      if (lx < F::TX && gi <= n0)
        for (int ly = warp; ly < F::TY; ly += F::WARPS) {
          const int j = gy0 + F::H + ly;
          if (j > n1) break;
          const int srow = (F::H + ly) * F::RX + F::H;
          T* r0 = o0 + (int64_t)j * P.sy;
          T* r1 = o1 + (int64_t)j * P.sy;
          if (!edge_tile && gi + 1 <= n0) {
            *reinterpret_cast<V*>(r0 + gi) = *reinterpret_cast<const V*>(s0 + srow + lx);
            *reinterpret_cast<V*>(r1 + gi) = *reinterpret_cast<const V*>(s1 + srow + lx);
            continue;
          }
          for (int d = 0; d < 2; ++d) {
            const int i = gi + d;
            if (i > n0) break;
            const T v0 = s0[srow + lx + d], v1 = s1[srow + lx + d];
            r0[i] = v0;
            r1[i] = v1;
            if (P.wt && near_boundary(P, i, j, 0, 2)) write_through<T, 2>(P, o0, o1, i, j, 0, v0, v1);
          }
        }
    }
    __syncthreads();  // the buffer is refilled for a later tile
    if (NBUF == 1 && nxt < n && tid == 0) issue(nxt, 0);
    cur = nxt;
    if (NBUF == 2) buf ^= 1;
  }
}

}  // namespace bsam
