// amr.cuh -- ghost cells of refined (AMR) patches and FillDown, 2D, FP64.
//
// Above the root level SetGhost (boundary.f90:58-89) fills a patch's ghost
// ring in three ordered steps, one launch each over all patches of the level:
//   k_interp2      coarse-fine interpolation on internal faces
//                  (InterpolateCoarseFine -> Interpolate2D, boundary.f90:91-323)
//   k_overlap      sibling exchange (ApplyOnLevelPairs -> TransferBC ->
//                  GhostOverlap, boundary.f90:325-415)
//   k_setbc_list   physical faces (SetBC2D, boundary.f90:643-744)
// Each step reads interior cells (or, for SetBC, ghosts the earlier steps
// wrote) and writes ghosts only, so cells within a step are independent.
#pragma once
#include "kernels.cuh"

namespace bsam {

// Boundary module coefficients (boundary.f90:45-54; FP64 under the
// reference's -fdefault-real-8 build).
constexpr double kA1 = -(1.0 / 5.0), kA2 = 2.0 / 3.0, kA3 = 8.0 / 15.0;
constexpr double kB1 = 5.0 / 32.0, kB2 = 15.0 / 16.0, kB3 = -(3.0 / 32.0);

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
__device__ void interp2_ghost(const DevPatch& P, const DevPatch& R, int ipass, int gi, int gj) {
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

// One CTA per patch of the list; threads over the 2(m1 + 2) + 2 m2 ring cells.
__global__ void k_interp2(const DevPatch* __restrict__ PT, const int* __restrict__ patches,
                          int ipass) {
  const DevPatch P = PT[patches[blockIdx.x]];
  const DevPatch R = PT[P.parent];
  const int m1 = P.n[0], m2 = P.n[1];
  const int nring = 2 * (m1 + 2) + 2 * m2;
  for (int g = threadIdx.x; g < nring; g += blockDim.x) {
    int gi, gj;
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
    interp2_ghost(P, R, ipass, gi, gj);
  }
}

// One GhostOverlap transfer: dst(i, j) = src(i + di, j + dj) over the
// dst-local box [i0, i1] x [j0, j1] (src cells are interior cells).
struct OverlapCopy {
  int32_t dst, src, i0, i1, j0, j1, di, dj;
};

__global__ void k_overlap(const DevPatch* __restrict__ PT, const OverlapCopy* __restrict__ cps) {
  const OverlapCopy o = cps[blockIdx.x];
  const DevPatch D = PT[o.dst];
  const DevPatch S = PT[o.src];
  const int w = o.i1 - o.i0 + 1, hgt = o.j1 - o.j0 + 1;
  for (int e = threadIdx.x; e < w * hgt; e += blockDim.x) {
    const int i = o.i0 + e % w, j = o.j0 + e / w;
#pragma unroll
    for (int v = 0; v < 2; ++v)
      fld<double>(D.q[v])[cidx(D, i, j, 0)] = fld<double>(S.q[v])[cidx(S, i + o.di, j + o.dj, 0)];
  }
}

// SetBC on every patch of a list (one CTA per patch), the k_setbc rule: a
// ghost outside in the physical dimensions S takes the face maps of S applied
// to the cell reflected across S (cells outside only in internal dimensions
// are left as the earlier steps wrote them).
template <int D>
__global__ void k_setbc_list(const DevPatch* __restrict__ PT, const int* __restrict__ patches) {
  const DevPatch P = PT[patches[blockIdx.x]];
  const int e0 = P.n[0] + 2, e1 = P.n[1] + 2;
  const int64_t total = (int64_t)e0 * e1 * (D == 3 ? P.n[2] + 2 : 1);
  for (int64_t g = threadIdx.x; g < total; g += blockDim.x) {
    int co[3] = {(int)(g % e0), (int)((g / e0) % e1), D == 3 ? (int)(g / ((int64_t)e0 * e1)) : 0};
    int src[3] = {co[0], co[1], co[2]};
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
    if (!write) continue;
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
}

// FillDownLevel for the solution (afas:241-310): parent%q(mb) = Restriction(q)
// over the footprint tiles of a level (q only; ghosts of a physical parent by
// write-through, those of a refined parent by its SetGhost afterwards).
__global__ void __launch_bounds__(BLOCK_THREADS)
    k_filldown2(const DevPatch* __restrict__ PT, const Item* __restrict__ items) {
  const Item it = items[blockIdx.x];
  const DevPatch C = PT[it.patch];
  const DevPatch P = PT[C.parent];
  const int jc = it.ty * TILE_Y + threadIdx.y + 1;
  if (jc > C.cn[1]) return;
  const int ic0 = (it.tx * 32 + threadIdx.x) * 2 + 1;
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    const int ic = ic0 + t;
    if (ic > C.cn[0]) break;
    const int i = 2 * ic, j = 2 * jc;
    double val[2];
#pragma unroll
    for (int v = 0; v < 2; ++v) {
      const double* a = fld<double>(C.q[v]);
      val[v] = 0.25 * (a[cidx(C, i, j, 0)] + a[cidx(C, i - 1, j, 0)] + a[cidx(C, i, j - 1, 0)] +
                       a[cidx(C, i - 1, j - 1, 0)]);
    }
    const int pi = C.off[0] + ic, pj = C.off[1] + jc;
    double* p0 = fld<double>(P.q[0]);
    double* p1 = fld<double>(P.q[1]);
    const int64_t pc = cidx(P, pi, pj, 0);
    p0[pc] = val[0];
    p1[pc] = val[1];
    if (P.wt && near_boundary(P, pi, pj, 0, 2))
      write_through<double, 2>(P, p0, p1, pi, pj, 0, val[0], val[1]);
  }
}

}  // namespace bsam
