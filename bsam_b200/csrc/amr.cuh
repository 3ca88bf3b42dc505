// amr.cuh -- ghost cells of refined (AMR) patches and FillDown, FP64.
//
// Above the root level SetGhost (boundary.f90:58-89) fills a patch's ghost
// ring in three ordered steps, done for each patch by one CTA of a single
// launch over the level (k_ghost2 / k_ghost3):
//   interpolation  coarse-fine interpolation on internal faces
//                  (InterpolateCoarseFine -> Interpolate2D / Interpolate3D,
//                  boundary.f90:91-323, 1299-1799)
//   overlap        sibling exchange (ApplyOnLevelPairs -> TransferBC ->
//                  GhostOverlap, boundary.f90:325-415)
//   SetBC          physical faces (SetBC2D/3D, boundary.f90:643-891)
// Each step reads interior cells (or, for SetBC, ghosts the earlier steps
// wrote) and writes ghosts only, so cells within a step are independent.
#pragma once
#include "kernels.cuh"

namespace bsam {

// Boundary module coefficients (boundary.f90:45-54; FP64 under the
// reference's -fdefault-real-8 build).
constexpr double kA1 = -(1.0 / 5.0), kA2 = 2.0 / 3.0, kA3 = 8.0 / 15.0;
constexpr double kB1 = 5.0 / 32.0, kB2 = 15.0 / 16.0, kB3 = -(3.0 / 32.0);
constexpr double kC1 = 9.0 / 16.0, kC2 = 3.0 / 16.0, kC3 = 3.0 / 16.0, kC4 = 1.0 / 16.0;

// One ghost of Interpolate2D: g = a1*q(f2) + a2*q(f1) + a3*coarse, where
// coarse is either one parent value or the three-point fit along the face.
__device__ __forceinline__ double interp_value(double f2, double f1, double c) {
  return kA1 * f2 + kA2 * f1 + kA3 * c;
}
__device__ __forceinline__ double face_fit(double c1, double c2, double c3) {
  return kB1 * c1 + kB2 * c2 + kB3 * c3;
}

// Ghost (gi, gj) of patch P for colour pass ipass (1 red, 2 black, 0 both);
// parent R.  Positions follow Interpolate2D statement by statement: the four
// corners always, face ghosts on internal faces only.
static __device__ void interp2_ghost(const DevPatch& P, const DevPatch& R, int ipass, int gi, int gj) {
  const int m1 = P.n[0], m2 = P.n[1];
  // Parent index box of the patch (mbounds): off + 1 .. off + cn.
  const int b11 = P.off[0] + 1, b12 = P.off[0] + P.cn[0];
  const int b21 = P.off[1] + 1, b22 = P.off[1] + P.cn[1];
  const bool red = ipass == 1 || ipass == 0, black = ipass == 2 || ipass == 0;
  const bool f1 = P.bc[0] == BC_NONE, f2 = P.bc[1] == BC_NONE;
  const bool f3 = P.bc[2] == BC_NONE, f4 = P.bc[3] == BC_NONE;
#pragma unroll
  for (int v = 0; v < 2; ++v) {
    const double* q = fld<double>(P.q[v]);
    const double* c = fld<double>(R.q[v]);
    auto Q = [&](int i, int j) { return q[cidx(P, i, j, 0)]; };
    auto C = [&](int i, int j) { return c[cidx(R, i, j, 0)]; };
    double val = 0.0;
    bool set = false;
    if (gi == m1 + 1 && gj == m2 + 1) {
      if (red) { val = interp_value(Q(m1 - 1, m2 - 1), Q(m1, m2), C(b12 + 1, b22 + 1)); set = true; }
    } else if (gi == 0 && gj == 0) {
      if (red) { val = interp_value(Q(2, 2), Q(1, 1), C(b11 - 1, b21 - 1)); set = true; }
    } else if (gi == m1 + 1 && gj == 0) {
      if (black) { val = interp_value(Q(m1 - 1, 2), Q(m1, 1), C(b12 + 1, b21 - 1)); set = true; }
    } else if (gi == 0 && gj == m2 + 1) {
      if (black) { val = interp_value(Q(2, m2 - 1), Q(1, m2), C(b11 - 1, b22 + 1)); set = true; }
    } else if (gi == 0) {  // face 1, j in 1..m2
      const int j = gj;
      if (!f1) return;
      if ((j & 1) == 0 && red) {
        set = true;
        if (j < m2) val = interp_value(Q(2, j + 2), Q(1, j + 1), C(b11 - 1, b21 + (j - 2) / 2));
        else val = interp_value(Q(2, m2), Q(1, m2),
                                face_fit(C(b11 - 1, b22 + 1), C(b11 - 1, b22), C(b11 - 1, b22 - 1)));
      } else if ((j & 1) == 1 && black) {
        set = true;
        if (j > 1) val = interp_value(Q(2, j - 2), Q(1, j - 1), C(b11 - 1, b21 + 1 + (j - 3) / 2));
        else val = interp_value(Q(2, 1), Q(1, 1),
                                face_fit(C(b11 - 1, b21 - 1), C(b11 - 1, b21), C(b11 - 1, b21 + 1)));
      }
    } else if (gi == m1 + 1) {  // face 2
      const int j = gj;
      if (!f2) return;
      if ((j & 1) == 1 && red) {
        set = true;
        if (j > 1) val = interp_value(Q(m1 - 1, j - 2), Q(m1, j - 1), C(b12 + 1, b21 + 1 + (j - 3) / 2));
        else val = interp_value(Q(m1 - 1, 1), Q(m1, 1),
                                face_fit(C(b12 + 1, b21 - 1), C(b12 + 1, b21), C(b12 + 1, b21 + 1)));
      } else if ((j & 1) == 0 && black) {
        set = true;
        if (j < m2) val = interp_value(Q(m1 - 1, j + 2), Q(m1, j + 1), C(b12 + 1, b21 + (j - 2) / 2));
        else val = interp_value(Q(m1 - 1, m2), Q(m1, m2),
                                face_fit(C(b12 + 1, b22 + 1), C(b12 + 1, b22), C(b12 + 1, b22 - 1)));
      }
    } else if (gj == 0) {  // face 3, i in 1..m1
      const int i = gi;
      if (!f3) return;
      if ((i & 1) == 0 && red) {
        set = true;
        if (i < m1) val = interp_value(Q(i + 2, 2), Q(i + 1, 1), C(b11 + (i - 2) / 2, b21 - 1));
        else val = interp_value(Q(m1, 2), Q(m1, 1),
                                face_fit(C(b12 + 1, b21 - 1), C(b12, b21 - 1), C(b12 - 1, b21 - 1)));
      } else if ((i & 1) == 1 && black) {
        set = true;
        if (i > 1) val = interp_value(Q(i - 2, 2), Q(i - 1, 1), C(b11 + 1 + (i - 3) / 2, b21 - 1));
        else val = interp_value(Q(1, 2), Q(1, 1),
                                face_fit(C(b11 - 1, b21 - 1), C(b11, b21 - 1), C(b11 + 1, b21 - 1)));
      }
    } else if (gj == m2 + 1) {  // face 4
      const int i = gi;
      if (!f4) return;
      if ((i & 1) == 1 && red) {
        set = true;
        if (i > 1) val = interp_value(Q(i - 2, m2 - 1), Q(i - 1, m2), C(b11 + 1 + (i - 3) / 2, b22 + 1));
        else val = interp_value(Q(1, m2 - 1), Q(1, m2),
                                face_fit(C(b11 - 1, b22 + 1), C(b11, b22 + 1), C(b11 + 1, b22 + 1)));
      } else if ((i & 1) == 0 && black) {
        set = true;
        if (i < m1) val = interp_value(Q(i + 2, m2 - 1), Q(i + 1, m2), C(b11 + (i - 2) / 2, b22 + 1));
        else val = interp_value(Q(m1, m2 - 1), Q(m1, m2),
                                face_fit(C(b12 + 1, b22 + 1), C(b12, b22 + 1), C(b12 - 1, b22 + 1)));
      }
    }
    if (set) fld<double>(P.q[v])[cidx(P, gi, gj, 0)] = val;
  }
}

// Ghost (g0, g1, g2) of 3D patch P for colour pass ipass (1 red, 2 black,
// 0 both); parent R.  Every statement of Interpolate3D writes ghosts only and
// reads interior fine cells and parent cells only, so a ghost's value is that
// of the last statement writing it, evaluated here from the ghost's position:
//   3 coordinates outside  corner   (boundary.f90:1322-1342)
//   2 outside              edge     (1344-1478)
//   1 outside              face     (1480-1797), internal faces only: yellow
//                          (even, even) and blue (odd, odd) cells in one
//                          colour, green (odd, even) and red (even, odd) in
//                          the other, the face's four corner cells always.
// Corners and edges are skipped in the red pass when one of their faces is
// physical; for the edges along y the z face passes that check only with code
// 2 or 99 (boundary.f90:1354 compares with 99, not 999), kept as written.
static __device__ void interp3_ghost(const DevPatch& P, const DevPatch& R, int ipass, int g0, int g1,
                              int g2) {
  const int m[3] = {P.n[0], P.n[1], P.n[2]};
  const int g[3] = {g0, g1, g2};
  int lo[3], hi[3], par[3], nout = 0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    lo[d] = P.off[d] + 1;  // the patch's footprint in the parent: mbounds
    hi[d] = P.off[d] + P.cn[d];
    par[d] = g[d] == 0 ? 1 : (g[d] == m[d] + 1 ? 2 : 0);
    nout += par[d] != 0;
  }
  // GetFaceIndex (boundary.f90:1271-1297) of an outside dimension.
  auto fs = [&](int d) { return par[d] == 1 ? 2 : m[d] - 1; };
  auto ff = [&](int d) { return par[d] == 1 ? 1 : m[d]; };
  auto fp = [&](int d) { return par[d] == 1 ? lo[d] - 1 : hi[d] + 1; };
  auto face = [&](int d) { return 2 * d + par[d] - 1; };
  auto internal = [&](int f) { return P.code[f] == 2 || P.code[f] == 999; };
  auto edge_y_keeps_z = [&](int f) { return P.code[f] == 2 || P.code[f] == 99; };
  if (nout == 0) return;
  if (nout == 3) {
    if (ipass == 1 && !(internal(face(0)) && internal(face(1)) && internal(face(2)))) return;
  } else if (nout == 2) {
    if (ipass == 1) {
      if (par[1] == 0 && !(internal(face(0)) && edge_y_keeps_z(face(2)))) return;
      if (par[2] == 0 && !(internal(face(0)) && internal(face(1)))) return;
      if (par[0] == 0 && !(internal(face(1)) && internal(face(2)))) return;
    }
  } else {
    int d = par[0] ? 0 : (par[1] ? 1 : 2);
    if (!internal(face(d))) return;
  }
#pragma unroll
  for (int v = 0; v < 2; ++v) {
    const double* q = fld<double>(P.q[v]);
    const double* c = fld<double>(R.q[v]);
    auto Q = [&](const int* x) { return q[cidx(P, x[0], x[1], x[2])]; };
    auto C = [&](const int* x) { return c[cidx(R, x[0], x[1], x[2])]; };
    // Second (S) and first (F) fine sources and the parent index (X) in the
    // outside dimensions; the others are set per case below.
    int S[3], F[3], X[3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
      if (par[d]) {
        S[d] = fs(d);
        F[d] = ff(d);
        X[d] = fp(d);
      }
    // The three-point fit along dimension d at parent indices k0, k1, k2.
    auto fit = [&](int d, int k0, int k1, int k2) {
      int Y[3] = {X[0], X[1], X[2]};
      Y[d] = k0;
      const double a = C(Y);
      Y[d] = k1;
      const double b = C(Y);
      Y[d] = k2;
      const double e = C(Y);
      return kB1 * a + kB2 * b + kB3 * e;
    };
    double par_v;
    if (nout == 3) {
      par_v = C(X);
    } else if (nout == 2) {
      const int e = par[0] == 0 ? 0 : (par[1] == 0 ? 1 : 2);
      const int t = g[e], me = m[e];
      if (t == 1) {
        S[e] = F[e] = 1;
        par_v = fit(e, lo[e] - 1, lo[e], lo[e] + 1);
      } else if (t == me) {
        S[e] = F[e] = me;
        par_v = fit(e, hi[e] + 1, hi[e], hi[e] - 1);
      } else if (t & 1) {  // 3:me-1:2
        S[e] = t - 2;
        F[e] = t - 1;
        X[e] = lo[e] + (t - 1) / 2;
        par_v = C(X);
      } else {  // 2:me-2:2
        S[e] = t + 2;
        F[e] = t + 1;
        X[e] = lo[e] + t / 2 - 1;
        par_v = C(X);
      }
    } else {
      const int d = par[0] ? 0 : (par[1] ? 1 : 2);
      const int u = d == 0 ? 1 : 0, w = d == 2 ? 1 : 2;
      const int tu = g[u], tw = g[w], mu = m[u], mw = m[w];
      const bool cu = tu == 1 || tu == mu, cw = tw == 1 || tw == mw;
      const int p = par[d];
      const bool col_a = ipass == 0 || (p + ipass) % 2 == 0;  // yellow, blue
      const bool col_b = ipass == 0 || (p + ipass) % 2 == 1;  // green, red
      // Source and parent indices along u (or w) for a cell t of the section:
      // odd t >= 3 from the diagonal below, even t <= m - 2 from above.
      auto along = [&](int x, int t, int lo_x) {
        if (t & 1) {
          S[x] = t - 2;
          F[x] = t - 1;
          X[x] = lo_x + (t - 1) / 2;
        } else {
          S[x] = t + 2;
          F[x] = t + 1;
          X[x] = lo_x + t / 2 - 1;
        }
      };
      if (cu && cw) {  // the face's corner cells (four-point fit)
        S[u] = F[u] = tu;
        S[w] = F[w] = tw;
        const int bu = tu == 1 ? lo[u] : hi[u], pu = tu == 1 ? lo[u] - 1 : hi[u] + 1;
        const int bw = tw == 1 ? lo[w] : hi[w], pw = tw == 1 ? lo[w] - 1 : hi[w] + 1;
        int Y[3] = {X[0], X[1], X[2]};
        Y[u] = bu;
        Y[w] = bw;
        const double k1 = C(Y);
        Y[u] = pu;
        const double k2 = C(Y);
        Y[u] = bu;
        Y[w] = pw;
        const double k3 = C(Y);
        Y[u] = pu;
        const double k4 = C(Y);
        par_v = kC1 * k1 + kC2 * k2 + kC3 * k3 + kC4 * k4;
      } else {
        const bool eu = (tu & 1) == 0, ew = (tw & 1) == 0;
        if (!((eu == ew) ? col_a : col_b)) return;
        if (tu == 1 || tu == mu) {  // strip along w at the u edge of the face
          S[u] = F[u] = tu;
          along(w, tw, lo[w]);
          par_v = tu == 1 ? fit(u, lo[u] - 1, lo[u], lo[u] + 1) : fit(u, hi[u] + 1, hi[u], hi[u] - 1);
        } else if (tw == 1 || tw == mw) {  // strip along u at the w edge
          S[w] = F[w] = tw;
          along(u, tu, lo[u]);
          par_v = tw == 1 ? fit(w, lo[w] - 1, lo[w], lo[w] + 1) : fit(w, hi[w] + 1, hi[w], hi[w] - 1);
        } else {  // the face's interior section
          along(u, tu, lo[u]);
          along(w, tw, lo[w]);
          par_v = C(X);
        }
      }
    }
    const double val = kA1 * Q(S) + kA2 * Q(F) + kA3 * par_v;
    fld<double>(P.q[v])[cidx(P, g0, g1, g2)] = val;
  }
}

// One GhostOverlap transfer: dst(i, j, k) = src(i + di, j + dj, k + dk) over
// the dst-local box [i0, i1] x [j0, j1] x [k0, k1] (k0 = k1 = 0, dk = 0 in
// 2D; src cells are interior cells).
struct OverlapCopy {
  int32_t dst, src, i0, i1, j0, j1, k0, k1, di, dj, dk;
};

// SetBC at one ring cell (g0, g1, g2) of patch P: a ghost outside in the
// physical dimensions S takes the face maps of S applied to the cell
// reflected across S (cells outside only in internal dimensions are left as
// the interpolation and the sibling copies wrote them).
template <int D>
__device__ __forceinline__ void setbc_cell(const DevPatch& P, int g0, int g1, int g2) {
  const int co[3] = {g0, g1, g2};
  int src[3] = {g0, g1, g2};
  int codes[3] = {BC_NONE, BC_NONE, BC_NONE};
  bool write = false;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    if (co[d] == 0 && P.bc[2 * d] != BC_NONE) {
      src[d] = 1;
      codes[d] = P.bc[2 * d];
      write = true;
    } else if (co[d] == P.n[d] + 1 && P.bc[2 * d + 1] != BC_NONE) {
      src[d] = P.n[d];
      codes[d] = P.bc[2 * d + 1];
      write = true;
    }
  }
  if (!write) return;
#pragma unroll
  for (int v = 0; v < 2; ++v) {
    double* q = fld<double>(P.q[v]);
    double val = q[cidx(P, src[0], src[1], src[2])];
#pragma unroll
    for (int d = 0; d < D; ++d)
      if (codes[d] != BC_NONE) val = bc_map<double>(codes[d], val);
    q[cidx(P, co[0], co[1], co[2])] = val;
  }
}

// The 2D ring cell g of a patch with m1 x m2 interior cells (bottom row, top
// row, left column, right column).
__device__ __forceinline__ void ring2(int g, int m1, int m2, int& gi, int& gj) {
  if (g < m1 + 2) {
    gi = g;
    gj = 0;
  } else if (g < 2 * (m1 + 2)) {
    gi = g - (m1 + 2);
    gj = m2 + 1;
  } else if (g < 2 * (m1 + 2) + m2) {
    gi = 0;
    gj = g - 2 * (m1 + 2) + 1;
  } else {
    gi = m1 + 1;
    gj = g - 2 * (m1 + 2) - m2 + 1;
  }
}

// SetGhost of a 2D refined level in one launch, one CTA per patch: the
// patch's coarse-fine interpolation (interp2_ghost on every ring cell), then
// the sibling copies into its ring (the overlap entries whose dst is this
// patch: ranges[b] = {first, count} into the list sorted by dst), then its
// physical faces (setbc_cell).  Each step writes only this patch's ring and reads the
// parent, this patch, and siblings' interiors, which no CTA writes here, so
// the CTA barrier between the steps orders everything that depends on them.
// The body is shared with the batch's list kernel (kb_ghost): patch p's
// transfers are cps[rg.x, rg.x + rg.y).  Every thread of the CTA calls it.
__device__ __forceinline__ void ghost2_patch(const DevPatch* __restrict__ PT, int p,
                                             const OverlapCopy* __restrict__ cps, int2 rg,
                                             int ipass) {
  // The records are read in place (L1-cached), not copied: a copy of two
  // records held 192 registers and limited the launch to two CTAs per SM.
  const DevPatch& P = PT[p];
  const DevPatch& R = PT[P.parent];
  const int m1 = P.n[0], m2 = P.n[1];
  const int nring = 2 * (m1 + 2) + 2 * m2;
  for (int g = threadIdx.x; g < nring; g += blockDim.x) {
    int gi, gj;
    ring2(g, m1, m2, gi, gj);
    interp2_ghost(P, R, ipass, gi, gj);
  }
  __syncthreads();
  // Sibling copies, a warp per copy: the strips are a few dozen cells, and
  // each copy starts with a chain of dependent reads (the copy, the
  // sibling's record), so the warps run their chains side by side.  The
  // siblings are disjoint, so no ghost is written by two copies and the
  // order of the copies does not matter.
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int c = rg.x + (int)(threadIdx.x >> 5); c < rg.x + rg.y; c += nw) {
    const OverlapCopy o = cps[c];
    const DevPatch& S = PT[o.src];
    const int w = o.i1 - o.i0 + 1, hgt = o.j1 - o.j0 + 1;
    for (int e = lane; e < w * hgt; e += 32) {
      const int i = o.i0 + e % w, j = o.j0 + e / w;
#pragma unroll
      for (int v = 0; v < 2; ++v)
        fld<double>(P.q[v])[cidx(P, i, j, 0)] = fld<double>(S.q[v])[cidx(S, i + o.di, j + o.dj, 0)];
    }
  }
  __syncthreads();
  for (int g = threadIdx.x; g < nring; g += blockDim.x) {
    int gi, gj;
    ring2(g, m1, m2, gi, gj);
    setbc_cell<2>(P, gi, gj, 0);
  }
}

static __global__ void k_ghost2(const DevPatch* __restrict__ PT, const int* __restrict__ patches,
                         const OverlapCopy* __restrict__ cps, const int2* __restrict__ ranges,
                         int ipass) {
  ghost2_patch(PT, patches[blockIdx.x], cps, ranges[blockIdx.x], ipass);
}

// The 3D ring cell g of a patch with m1 x m2 x m3 interior cells, in
// order: the two k planes, then the 2D ring of each interior plane.
__device__ __forceinline__ void ring3(int g, int m1, int m2, int m3, int& gi, int& gj, int& gk) {
  const int plane = (m1 + 2) * (m2 + 2), rg2 = 2 * (m1 + 2) + 2 * m2;
  if (g < 2 * plane) {
    gk = g < plane ? 0 : m3 + 1;
    const int r = g % plane;
    gi = r % (m1 + 2);
    gj = r / (m1 + 2);
  } else {
    const int r0 = g - 2 * plane;
    gk = 1 + r0 / rg2;
    ring2(r0 % rg2, m1, m2, gi, gj);
  }
}

// SetGhost of a 3D refined level in one launch: k_ghost2's structure with
// Interpolate3D (interp3_ghost), the 3D overlap boxes and the 3D face rule.
__device__ __forceinline__ void ghost3_patch(const DevPatch* __restrict__ PT, int p,
                                             const OverlapCopy* __restrict__ cps, int2 rg,
                                             int ipass) {
  // The records are read in place (L1-cached), not copied: a copy of two
  // records held 192 registers and limited the launch to two CTAs per SM.
  const DevPatch& P = PT[p];
  const DevPatch& R = PT[P.parent];
  const int m1 = P.n[0], m2 = P.n[1], m3 = P.n[2];
  const int nring = 2 * (m1 + 2) * (m2 + 2) + m3 * (2 * (m1 + 2) + 2 * m2);
  for (int g = threadIdx.x; g < nring; g += blockDim.x) {
    int gi, gj, gk;
    ring3(g, m1, m2, m3, gi, gj, gk);
    interp3_ghost(P, R, ipass, gi, gj, gk);
  }
  __syncthreads();
  for (int c = rg.x; c < rg.x + rg.y; ++c) {
    const OverlapCopy o = cps[c];
    const DevPatch S = PT[o.src];
    const int w = o.i1 - o.i0 + 1, hgt = o.j1 - o.j0 + 1, dep = o.k1 - o.k0 + 1;
    for (int e = threadIdx.x; e < w * hgt * dep; e += blockDim.x) {
      const int i = o.i0 + e % w, j = o.j0 + (e / w) % hgt, k = o.k0 + e / (w * hgt);
#pragma unroll
      for (int v = 0; v < 2; ++v)
        fld<double>(P.q[v])[cidx(P, i, j, k)] =
            fld<double>(S.q[v])[cidx(S, i + o.di, j + o.dj, k + o.dk)];
    }
  }
  __syncthreads();
  for (int g = threadIdx.x; g < nring; g += blockDim.x) {
    int gi, gj, gk;
    ring3(g, m1, m2, m3, gi, gj, gk);
    setbc_cell<3>(P, gi, gj, gk);
  }
}

static __global__ void k_ghost3(const DevPatch* __restrict__ PT, const int* __restrict__ patches,
                         const OverlapCopy* __restrict__ cps, const int2* __restrict__ ranges,
                         int ipass) {
  ghost3_patch(PT, patches[blockIdx.x], cps, ranges[blockIdx.x], ipass);
}

// FillDownLevel for the solution (afas:241-310): parent%q(mb) = Restriction(q)
// over the footprint tiles of a level (q only; ghosts of a physical parent by
// write-through, those of a refined parent by its SetGhost afterwards).  The
// restriction sums the children in Restriction2D/3D's order.
template <int D>
__device__ __forceinline__ void filldown_item(const DevPatch* __restrict__ PT, const Item it) {
  const DevPatch C = PT[it.patch];
  const DevPatch P = PT[C.parent];
  const int jc = it.ty * TILE_Y + threadIdx.y + 1;
  const int kc = D == 3 ? it.tz + 1 : 0;
  if (jc > C.cn[1]) return;
  const int ic0 = (it.tx * 32 + threadIdx.x) * 2 + 1;
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    const int ic = ic0 + t;
    if (ic > C.cn[0]) break;
    const int i = 2 * ic, j = 2 * jc, k = 2 * kc;
    double val[2];
#pragma unroll
    for (int v = 0; v < 2; ++v) {
      const double* a = fld<double>(C.q[v]);
      if (D == 2)
        val[v] = 0.25 * (a[cidx(C, i, j, 0)] + a[cidx(C, i - 1, j, 0)] + a[cidx(C, i, j - 1, 0)] +
                         a[cidx(C, i - 1, j - 1, 0)]);
      else
        val[v] = 0.125 * (a[cidx(C, i, j, k)] + a[cidx(C, i - 1, j, k)] + a[cidx(C, i, j - 1, k)] +
                          a[cidx(C, i - 1, j - 1, k)] + a[cidx(C, i, j, k - 1)] +
                          a[cidx(C, i - 1, j, k - 1)] + a[cidx(C, i, j - 1, k - 1)] +
                          a[cidx(C, i - 1, j - 1, k - 1)]);
    }
    const int pi = C.off[0] + ic, pj = C.off[1] + jc, pk = D == 3 ? C.off[2] + kc : 0;
    double* p0 = fld<double>(P.q[0]);
    double* p1 = fld<double>(P.q[1]);
    const int64_t pc = cidx(P, pi, pj, pk);
    p0[pc] = val[0];
    p1[pc] = val[1];
    if (P.wt && near_boundary(P, pi, pj, pk, D))
      write_through<double, D>(P, p0, p1, pi, pj, pk, val[0], val[1]);
  }
}

template <int D>
__global__ void __launch_bounds__(BLOCK_THREADS)
    k_filldown(const DevPatch* __restrict__ PT, const Item* __restrict__ items) {
  filldown_item<D>(PT, items[blockIdx.x]);
}

}  // namespace bsam
