// problem_ch.cuh -- device twins of the simple_cahn-hilliard problem module.
//
// The reference's plugin API is the Fortran module `Problem`
// (problems/simple_cahn-hilliard/problem.f90), whose routines the multigrid
// library calls by fixed names (lib/afasroutines.f90:318,434,556,653,801;
// lib/boundary.f90:645,748).  Here the module is a trait type, CahnHilliard,
// whose static members carry the same names and formulas, evaluated per cell
// from its stencil neighbourhood; the kernels reach it as `Problem`
// (problem.cuh), the one compile-time choice of the problem module.
// Operation order follows the Fortran expressions left to right so that FP64
// results match the reference arithmetic bit for bit (the library is built
// with --fmad=false, so no multiply-add is contracted).
#pragma once

namespace bsam {

// Approximate reciprocal of the FP32 working levels (PTX rcp.approx.ftz.f32,
// maximum relative error 2^-23), one instruction; the scalar and the paired
// forms of the FP32 update both take it.
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

struct CahnHilliard {
  // The module's sizes as the reference's problem data declares them
  // (problemdata.dat: nrvars, maux; errortype 1 = the user tagging routine).
  static constexpr int nrvars = 2;
  static constexpr int maux = 0;
  static constexpr int errortype = 1;
  // The fused 2D stage may update two FP32 cells at once with paired
  // arithmetic (fused2.cuh, relax_pair_f32): this module's Newton step.
  static constexpr bool paired_f32 = true;

  // Mob, Dfe, Dfc, D2fc (problem.f90:760-813).
  template <class T> static __device__ __forceinline__ T Mob(T) { return T(1); }
  template <class T> static __device__ __forceinline__ T Dfe(T c, T alpha) {
    return (c - T(0.5)) * alpha / T(4);
  }
  template <class T> static __device__ __forceinline__ T Dfc(T c, T alpha) {
    T cmh = c - T(0.5);
    return cmh * cmh * cmh * alpha;
  }
  template <class T> static __device__ __forceinline__ T D2fc(T c, T alpha) {
    T cmh = c - T(0.5);
    return T(3) * cmh * cmh * alpha;
  }

  // Dfc(b + e) - Dfc(b) = alpha e (3 c^2 + 3 c e + e^2), c = b - 1/2: the
  // change of the convex part over a correction e, formed so that rounding
  // scales with e (the correction form of the mixed-precision inner cycle).
  template <class T> static __device__ __forceinline__ T DfcDelta(T b, T e, T alpha) {
    const T c = b - T(0.5);
    return alpha * e * (T(3) * c * c + T(3) * c * e + e * e);
  }


  // Neighbourhood of one cell: centre values and the -/+ neighbours per
  // dimension, for both components (phi = q(:,:,1), mu = q(:,:,2)).
  template <class T, int D> struct Stencil {
    T pc, mc;        // phi, mu at the cell
    T pm[D], pp[D];  // phi at i-1 / i+1 (per dimension)
    T mm[D], mp[D];  // mu  at i-1 / i+1
  };

  // One cell of RelaxGrid2D / RelaxGrid3D (problem.f90:192-213, 485-516): the
  // per-cell 2x2 Newton update of (phi, mu) solved by Cramer's rule.
  // tmp1 = dt/h^2, tmp2 = eps2/h^2, tmp3 = 2d*eps2/h^2.
  // DELTA = true: the stencil holds a correction e of the base state whose phi
  // at the cell is `base`; the same Newton step is taken on
  // L(base + e) - L(base) = f, with Dfc replaced by DfcDelta and D2fc taken at
  // base + e.  DELTA = false is the reference's update, operation for
  // operation.
  template <class T, int D, bool DELTA = false>
  static __device__ __forceinline__ void RelaxCell(const Stencil<T, D>& s, T f0, T f1, T tmp1,
                                                   T tmp2, T tmp3, T alpha, T& phi, T& mu,
                                                   T base = T(0)) {
    T m[2 * D];
#pragma unroll
    for (int d = 0; d < D; ++d) {
      m[2 * d] = Mob(T(0.5) * (s.pm[d] + s.pc));
      m[2 * d + 1] = Mob(T(0.5) * (s.pp[d] + s.pc));
    }
    T msum = m[0];
#pragma unroll
    for (int t = 1; t < 2 * D; ++t) msum = msum + m[t];
    const T a12 = tmp1 * msum;
    const T cfull = DELTA ? base + s.pc : s.pc;
    if constexpr (sizeof(T) == 4) {
      // FP32 working levels of the mixed form: the same Newton step with
      // contracted products and one approximate reciprocal (rcp_approx), since
      // these levels only smooth a correction whose FP64 defect is recomputed
      // exactly; the FP64 path below keeps the reference's operation order.
      // Every operation is an explicitly rounded one the compiler may not
      // contract, so it evaluates exactly this sequence -- the one the paired
      // FP32 form of the fused 2D stage (relax_pair_f32) evaluates too.
      const float cf = DELTA ? __fadd_rn(base, s.pc) : s.pc;
      const float cmh = __fadd_rn(cf, -0.5f);
      const float u = __fmul_rn(__fmul_rn(3.f, cmh), cmh);
      const T d2 = __fmul_rn(u, alpha);
      const T a21f = -d2 - tmp3;
      T smuf = m[0] * s.mm[0] + m[1] * s.mp[0];
#pragma unroll
      for (int d = 1; d < D; ++d) {
        smuf = smuf + m[2 * d] * s.mm[d];
        smuf = smuf + m[2 * d + 1] * s.mp[d];
      }
      T sphf = s.pp[0] + s.pm[0];
#pragma unroll
      for (int d = 1; d < D; ++d) {
        sphf = sphf + s.pp[d];
        sphf = sphf + s.pm[d];
      }
      T nlf;
      if constexpr (DELTA) {
        // DfcDelta(base, e) = alpha e (3 c^2 + 3 c e + e^2), c = base - 1/2.
        const float c = __fadd_rn(base, -0.5f), e = s.pc;
        const float c3 = __fmul_rn(3.f, c);
        const float poly =
            __fadd_rn(__fadd_rn(__fmul_rn(c3, c), __fmul_rn(c3, e)), __fmul_rn(e, e));
        nlf = __fmul_rn(__fmul_rn(alpha, e), poly);
      } else {
        nlf = Dfc(s.pc, alpha);
      }
      const T b1f = __fmaf_rn(tmp1, smuf, f0);
      const T b2f = __fmaf_rn(-tmp2, sphf, __fmaf_rn(-d2, s.pc, f1 + nlf));
      const T detf = __fmaf_rn(-a12, a21f, T(1));
      const T r = rcp_approx(detf);
      phi = __fmaf_rn(-a12, b2f, b1f) * r;
      mu = __fmaf_rn(-a21f, b1f, b2f) * r;
      return;
    }
    const T a21 = -D2fc(cfull, alpha) - tmp3;
    // b(1): f + tmp1*(m1*mu(i-1) + m2*mu(i+1) + m3*mu(j-1) + m4*mu(j+1) ...)
    T smu = m[0] * s.mm[0] + m[1] * s.mp[0];
#pragma unroll
    for (int d = 1; d < D; ++d) {
      smu = smu + m[2 * d] * s.mm[d];
      smu = smu + m[2 * d + 1] * s.mp[d];
    }
    const T b1 = f0 + tmp1 * smu;
    // b(2): f + Dfc - D2fc*phi - tmp2*(phi(i+1) + phi(i-1) + phi(j+1) + ...)
    T sph = s.pp[0] + s.pm[0];
#pragma unroll
    for (int d = 1; d < D; ++d) {
      sph = sph + s.pp[d];
      sph = sph + s.pm[d];
    }
    const T nl = DELTA ? DfcDelta(base, s.pc, alpha) : Dfc(s.pc, alpha);
    const T b2 = f1 + nl - D2fc(cfull, alpha) * s.pc - tmp2 * sph;
    const T det = T(1) - a12 * a21;
    phi = (b1 - a12 * b2) / det;
    mu = (b2 - a21 * b1) / det;
  }

  // One cell of Operator2D / Operator3D (problem.f90:250-256, 554-560) with
  // ULapMob (304-329, 607-642), UDiv and ULap (gridutilities.f90:42-87,
  // 345-404):
  //   res1 = phi - tmp1 * UDiv(Mob * grad mu)
  //   res2 = mu - Dfc(phi) + tmp2 * ULap(phi)
  // DELTA = true: L(base + e) - L(base) for a correction e (see RelaxCell).
  template <class T, int D, bool DELTA = false>
  static __device__ __forceinline__ void OperatorCell(const Stencil<T, D>& s, T tmp1, T tmp2,
                                                      T alpha, T& r0, T& r1, T base = T(0)) {
    T udiv = Mob(T(0.5) * (s.pp[0] + s.pc)) * (s.mp[0] - s.mc) -
             Mob(T(0.5) * (s.pc + s.pm[0])) * (s.mc - s.mm[0]);
#pragma unroll
    for (int d = 1; d < D; ++d) {
      udiv = udiv + Mob(T(0.5) * (s.pp[d] + s.pc)) * (s.mp[d] - s.mc);
      udiv = udiv - Mob(T(0.5) * (s.pc + s.pm[d])) * (s.mc - s.mm[d]);
    }
    r0 = s.pc - tmp1 * udiv;
    T lap = s.pp[0] + s.pm[0];
#pragma unroll
    for (int d = 1; d < D; ++d) {
      lap = lap + s.pp[d];
      lap = lap + s.pm[d];
    }
    lap = lap - T(2 * D) * s.pc;
    const T nl = DELTA ? DfcDelta(base, s.pc, alpha) : Dfc(s.pc, alpha);
    r1 = s.mc - nl + tmp2 * lap;
  }

  // Source2D/3D followed by UpdateSourceFunction (problem.f90:278-279,
  // 281-303; lib/afasroutines.f90:467-472): f = Source(qold) + SourceUpdate,
  // with SourceUpdate = 0 for this problem.
  template <class T>
  static __device__ __forceinline__ void SourceCell(T qold_phi, T alpha, T& f0, T& f1) {
    f0 = qold_phi + T(0);
    f1 = -Dfe(qold_phi, alpha) + T(0);
  }

  // Ff (problem.f90:769-780): alpha c^2 (c-1)^2 / 4, the bulk free energy of
  // AfterStep's energy integral.
  static __device__ __forceinline__ double Ff(double c, double alpha) {
    const double cm1 = c - 1.0;
    return c * c * cm1 * cm1 * alpha / 4.0;
  }

  // SetErrFlagsUser2D/3D's test (problem.f90:135-163, 425-452) on the
  // undivided central differences dc[d] = c(+1) - c(-1) of the cell:
  // |grad c| > tol.
  template <int D>
  static __device__ __forceinline__ bool TagCell(const double (&dc)[D], double tol) {
    double s = dc[0] * dc[0] + dc[1] * dc[1];
    if (D == 3) s = s + dc[D - 1] * dc[D - 1];
    return fabs(sqrt(s)) > tol;
  }
};  // struct CahnHilliard

}  // namespace bsam
