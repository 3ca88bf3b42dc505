// bsam_oracle.cpp -- CPU oracle for the BSAM FAS V-cycle (TEST INFRASTRUCTURE).
//
// A plain C++ restatement of the reference Fortran hot path for the
// simple_cahn-hilliard problem module.  Only tests/, __graft_entry__.smoke()
// and bench.py's cpu_baseline leg load this file's library; the product path
// (bsam_b200/, include/) never does.
//
// Parity pinning: PINNED bit for bit against fixtures made by executing the
// reference's own Fortran source with a Fortran-subset interpreter
// (tests/golden/, tests/test_golden_reference.py) -- the leaf routines and
// their composition (MultigridIterations, the V-cycle, SetGhost, FillDown,
// ErrorAFAS) on uniform 2D / 3D and refined 2D hierarchies.  Known-answer
// tests and invariants add to that (tests/test_oracle.py,
// tests/test_oracle_amr.py).
//
// Faithfulness rules followed throughout:
//  * every array statement evaluates its whole right-hand side before the
//    assignment (Fortran array semantics);
//  * expressions are evaluated left to right exactly as written in the
//    reference (no reassociation; build with -ffp-contract=off);
//  * reductions (sum) run sequentially in column-major order;
//  * statement order of the reference routines is kept, including the
//    numerically dead FillDown / UpdateSourceFunction passes.
#include "bsam_oracle.h"

#include <array>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <vector>

namespace {

// Fortran-style array with arbitrary lower bounds, up to 4 dimensions,
// column-major (first index fastest).
struct FArr {
  int lo[4] = {0, 0, 0, 0};
  int n[4] = {0, 0, 0, 0};
  long st[4] = {0, 0, 0, 0};
  std::vector<double> d;
  void alloc(int l0, int h0, int l1, int h1, int l2, int h2, int l3, int h3,
             double v = 0.0) {
    int l[4] = {l0, l1, l2, l3}, h[4] = {h0, h1, h2, h3};
    long s = 1;
    for (int a = 0; a < 4; ++a) {
      lo[a] = l[a];
      n[a] = h[a] - l[a] + 1;
      if (n[a] < 0) n[a] = 0;
      st[a] = s;
      s *= n[a];
    }
    d.assign((size_t)s, v);
  }
  inline long idx(int i, int j, int k, int v) const {
    return (long)(i - lo[0]) + st[1] * (j - lo[1]) + st[2] * (k - lo[2]) +
           st[3] * (v - lo[3]);
  }
  inline double& operator()(int i, int j, int k, int v) { return d[idx(i, j, k, v)]; }
  inline double operator()(int i, int j, int k, int v) const { return d[idx(i, j, k, v)]; }
  int hi(int a) const { return lo[a] + n[a] - 1; }
};

// The nodeinfo patch record (lib/nodeinfodef.f90:124-219), reduced to the
// components the hot path touches.
struct Patch {
  int level = 0, nrvars = 2, mbc = 1, maux = 0;
  int mx[3] = {1, 1, 1};
  int mbounds[3][2] = {{1, 1}, {1, 1}, {1, 1}};
  int mglobal[3][2] = {{1, 1}, {1, 1}, {1, 1}};
  int mthbc[6] = {1, 1, 1, 1, 1, 1};
  double dx[3] = {0, 0, 0}, xlower[3] = {0, 0, 0};
  bool tobedeleted = false;
  Patch* parent = nullptr;
  FArr q, qold, qc, f, rf, ftmp;
};

// Module state of NodeInfoDef / ProblemDef used on the hot path.
struct Ctx {
  int ndims = 2;
  double dt = 0, qerrortol = 1e-6, alpha = 1, eps = 0, eps2 = 0;
  int maxvcycles = 20, nsmoothingpasses = 2, errortype = 1;
  int minlevel = 0, finestlevel = 0;
  static const int rootlevel = 0;
  // periodicboundaryconditions (nodeinfodef.f90:50), set by PeriodicSetup
  // (boundary.f90:893-963) when a root face has code 2; qpo = 0
  // (bsamroutines.f90:241).
  bool periodic = false;
  std::vector<std::unique_ptr<Patch>> store;
  // levels[level - minlevel] in ApplyOnLevel order (youngest first).
  std::vector<std::vector<Patch*>> levels;
  std::vector<Patch*>& on(int level) { return levels[level - minlevel]; }
};

// ---------------------------------------------------------------------------
// Problem module elemental functions (problem.f90:760-813).
inline double Mob(const Ctx&, double) { return 1.0; }
inline double Ff(const Ctx& c, double x) {
  double cm1 = x - 1.0;
  return x * x * cm1 * cm1 * c.alpha / 4.0;
}
inline double Dfe(const Ctx& c, double x) { return (x - 0.5) * c.alpha / 4.0; }
inline double Dfc(const Ctx& c, double x) {
  double cmh = x - 0.5;
  return cmh * cmh * cmh * c.alpha;
}
inline double D2fc(const Ctx& c, double x) {
  double cmh = x - 0.5;
  return 3.0 * cmh * cmh * c.alpha;
}

// AllocFields (lib/bsamstorage.f90:46-123).
void AllocFields(const Ctx& c, Patch& p) {
  int mx[3] = {1, 1, 1}, cmx[3] = {1, 1, 1};
  for (int n = 0; n < c.ndims; ++n) {
    mx[n] = p.mx[n];
    cmx[n] = (mx[n] % 2 == 1) ? 1 : mx[n] / 2;
  }
  int m = p.mbc, nv = p.nrvars;
  if (c.ndims == 2) {
    p.q.alloc(1 - m, mx[0] + m, 1 - m, mx[1] + m, 1, 1, 1, nv);
    p.qold.alloc(1 - m, mx[0] + m, 1 - m, mx[1] + m, 1, 1, 1, nv);
    p.qc.alloc(1 - m, cmx[0] + m, 1 - m, cmx[1] + m, 1, 1, 1, nv);
    p.f.alloc(1, mx[0], 1, mx[1], 1, 1, 1, nv);
    p.rf.alloc(1, mx[0], 1, mx[1], 1, 1, 1, nv);
    p.ftmp.alloc(1, mx[0], 1, mx[1], 1, 1, 1, nv);
  } else {
    p.q.alloc(1 - m, mx[0] + m, 1 - m, mx[1] + m, 1 - m, mx[2] + m, 1, nv);
    p.qold.alloc(1 - m, mx[0] + m, 1 - m, mx[1] + m, 1 - m, mx[2] + m, 1, nv);
    p.qc.alloc(1 - m, cmx[0] + m, 1 - m, cmx[1] + m, 1 - m, cmx[2] + m, 1, nv);
    p.f.alloc(1, mx[0], 1, mx[1], 1, mx[2], 1, nv);
    p.rf.alloc(1, mx[0], 1, mx[1], 1, mx[2], 1, nv);
    p.ftmp.alloc(1, mx[0], 1, mx[1], 1, mx[2], 1, nv);
  }
}

// ---------------------------------------------------------------------------
// RelaxGrid2D (problem.f90:164-215).  q has bounds (0:mx+1), f (1:mx).
void RelaxGrid2D(const Ctx& c, FArr& q, const FArr& f, const int* mx, double h,
                 int ipass) {
  double h2 = h * h;
  double tmp1 = c.dt / h2;
  double tmp2 = c.eps2 / h2;
  double tmp3 = 4.0 * c.eps2 / h2;
  for (int j = 1; j <= mx[1]; ++j) {
    for (int i = 1 + (j + ipass) % 2; i <= mx[0]; i += 2) {
      double m1 = Mob(c, 0.5 * (q(i - 1, j, 1, 1) + q(i, j, 1, 1)));
      double m2 = Mob(c, 0.5 * (q(i + 1, j, 1, 1) + q(i, j, 1, 1)));
      double m3 = Mob(c, 0.5 * (q(i, j - 1, 1, 1) + q(i, j, 1, 1)));
      double m4 = Mob(c, 0.5 * (q(i, j + 1, 1, 1) + q(i, j, 1, 1)));
      double a12 = tmp1 * (m1 + m2 + m3 + m4);
      double a21 = -D2fc(c, q(i, j, 1, 1)) - tmp3;
      double b1 = f(i, j, 1, 1) + tmp1 * (m1 * q(i - 1, j, 1, 2) + m2 * q(i + 1, j, 1, 2) +
                                          m3 * q(i, j - 1, 1, 2) + m4 * q(i, j + 1, 1, 2));
      double b2 = f(i, j, 1, 2) + Dfc(c, q(i, j, 1, 1)) - D2fc(c, q(i, j, 1, 1)) * q(i, j, 1, 1) -
                  tmp2 * (q(i + 1, j, 1, 1) + q(i - 1, j, 1, 1) + q(i, j + 1, 1, 1) +
                          q(i, j - 1, 1, 1));
      double det = 1.0 - a12 * a21;
      q(i, j, 1, 1) = (b1 - a12 * b2) / det;
      q(i, j, 1, 2) = (b2 - a21 * b1) / det;
    }
  }
}

// RelaxGrid3D (problem.f90:453-518).
void RelaxGrid3D(const Ctx& c, FArr& q, const FArr& f, const int* mx, double h,
                 int ipass) {
  double h2 = h * h;
  double tmp1 = c.dt / h2;
  double tmp2 = c.eps2 / h2;
  double tmp3 = 6.0 * c.eps2 / h2;
  for (int k = 1; k <= mx[2]; ++k) {
    for (int j = 1; j <= mx[1]; ++j) {
      for (int i = 1 + (k + j + ipass) % 2; i <= mx[0]; i += 2) {
        double m1 = Mob(c, 0.5 * (q(i - 1, j, k, 1) + q(i, j, k, 1)));
        double m2 = Mob(c, 0.5 * (q(i + 1, j, k, 1) + q(i, j, k, 1)));
        double m3 = Mob(c, 0.5 * (q(i, j - 1, k, 1) + q(i, j, k, 1)));
        double m4 = Mob(c, 0.5 * (q(i, j + 1, k, 1) + q(i, j, k, 1)));
        double m5 = Mob(c, 0.5 * (q(i, j, k - 1, 1) + q(i, j, k, 1)));
        double m6 = Mob(c, 0.5 * (q(i, j, k + 1, 1) + q(i, j, k, 1)));
        double a12 = tmp1 * (m1 + m2 + m3 + m4 + m5 + m6);
        double a21 = -D2fc(c, q(i, j, k, 1)) - tmp3;
        double b1 = f(i, j, k, 1) + tmp1 * (m1 * q(i - 1, j, k, 2) + m2 * q(i + 1, j, k, 2) +
                                            m3 * q(i, j - 1, k, 2) + m4 * q(i, j + 1, k, 2) +
                                            m5 * q(i, j, k - 1, 2) + m6 * q(i, j, k + 1, 2));
        double b2 = f(i, j, k, 2) + Dfc(c, q(i, j, k, 1)) -
                    D2fc(c, q(i, j, k, 1)) * q(i, j, k, 1) -
                    tmp2 * (q(i + 1, j, k, 1) + q(i - 1, j, k, 1) + q(i, j + 1, k, 1) +
                            q(i, j - 1, k, 1) + q(i, j, k + 1, 1) + q(i, j, k - 1, 1));
        double det = 1.0 - a12 * a21;
        q(i, j, k, 1) = (b1 - a12 * b2) / det;
        q(i, j, k, 2) = (b2 - a21 * b1) / det;
      }
    }
  }
}

// Operator2D (problem.f90:231-257) with ULapMob2D (304-329), UDiv2D and
// ULap2D (gridutilities.f90:42-87).  q carries the ring (0:mx+1); res is
// returned with bounds (1:mx).
void Operator2D(const Ctx& c, const FArr& q, const int* mx, double h, FArr& res) {
  double h2 = h * h;
  double tmp1 = c.dt / h2;
  double tmp2 = c.eps2 / h2;
  int n1 = mx[0], n2 = mx[1];
  res.alloc(1, n1, 1, n2, 1, 1, 1, 2);
  // ULapMob2D flux arrays f1(0:mx1,1:mx2), f2(1:mx1,0:mx2).
  FArr f1, f2;
  f1.alloc(0, n1, 1, n2, 1, 1, 1, 1);
  f2.alloc(1, n1, 0, n2, 1, 1, 1, 1);
  for (int j = 1; j <= n2; ++j)
    for (int i = 0; i <= n1; ++i)
      f1(i, j, 1, 1) = Mob(c, 0.5 * (q(i + 1, j, 1, 1) + q(i, j, 1, 1))) *
                       (q(i + 1, j, 1, 2) - q(i, j, 1, 2));
  for (int j = 0; j <= n2; ++j)
    for (int i = 1; i <= n1; ++i)
      f2(i, j, 1, 1) = Mob(c, 0.5 * (q(i, j + 1, 1, 1) + q(i, j, 1, 1))) *
                       (q(i, j + 1, 1, 2) - q(i, j, 1, 2));
  for (int j = 1; j <= n2; ++j)
    for (int i = 1; i <= n1; ++i) {
      double udiv = f1(i, j, 1, 1) - f1(i - 1, j, 1, 1) + f2(i, j, 1, 1) - f2(i, j - 1, 1, 1);
      res(i, j, 1, 1) = q(i, j, 1, 1) - tmp1 * udiv;
    }
  for (int j = 1; j <= n2; ++j)
    for (int i = 1; i <= n1; ++i) {
      double ulap = q(i + 1, j, 1, 1) + q(i - 1, j, 1, 1) + q(i, j + 1, 1, 1) +
                    q(i, j - 1, 1, 1) - 4.0 * q(i, j, 1, 1);
      res(i, j, 1, 2) = q(i, j, 1, 2) - Dfc(c, q(i, j, 1, 1)) + tmp2 * ulap;
    }
}

// Operator3D (problem.f90:534-561) with ULapMob3D (607-642), UDiv3D and
// ULap3D (gridutilities.f90:345-404).
void Operator3D(const Ctx& c, const FArr& q, const int* mx, double h, FArr& res) {
  double h2 = h * h;
  double tmp1 = c.dt / h2;
  double tmp2 = c.eps2 / h2;
  int n1 = mx[0], n2 = mx[1], n3 = mx[2];
  res.alloc(1, n1, 1, n2, 1, n3, 1, 2);
  FArr f1, f2, f3;
  f1.alloc(0, n1, 1, n2, 1, n3, 1, 1);
  f2.alloc(1, n1, 0, n2, 1, n3, 1, 1);
  f3.alloc(1, n1, 1, n2, 0, n3, 1, 1);
  for (int k = 1; k <= n3; ++k)
    for (int j = 1; j <= n2; ++j)
      for (int i = 0; i <= n1; ++i)
        f1(i, j, k, 1) = Mob(c, 0.5 * (q(i + 1, j, k, 1) + q(i, j, k, 1))) *
                         (q(i + 1, j, k, 2) - q(i, j, k, 2));
  for (int k = 1; k <= n3; ++k)
    for (int j = 0; j <= n2; ++j)
      for (int i = 1; i <= n1; ++i)
        f2(i, j, k, 1) = Mob(c, 0.5 * (q(i, j + 1, k, 1) + q(i, j, k, 1))) *
                         (q(i, j + 1, k, 2) - q(i, j, k, 2));
  for (int k = 0; k <= n3; ++k)
    for (int j = 1; j <= n2; ++j)
      for (int i = 1; i <= n1; ++i)
        f3(i, j, k, 1) = Mob(c, 0.5 * (q(i, j, k + 1, 1) + q(i, j, k, 1))) *
                         (q(i, j, k + 1, 2) - q(i, j, k, 2));
  for (int k = 1; k <= n3; ++k)
    for (int j = 1; j <= n2; ++j)
      for (int i = 1; i <= n1; ++i) {
        double udiv = f1(i, j, k, 1) - f1(i - 1, j, k, 1) + f2(i, j, k, 1) - f2(i, j - 1, k, 1) +
                      f3(i, j, k, 1) - f3(i, j, k - 1, 1);
        res(i, j, k, 1) = q(i, j, k, 1) - tmp1 * udiv;
      }
  for (int k = 1; k <= n3; ++k)
    for (int j = 1; j <= n2; ++j)
      for (int i = 1; i <= n1; ++i) {
        double ulap = q(i + 1, j, k, 1) + q(i - 1, j, k, 1) + q(i, j + 1, k, 1) +
                      q(i, j - 1, k, 1) + q(i, j, k + 1, 1) + q(i, j, k - 1, 1) -
                      6.0 * q(i, j, k, 1);
        res(i, j, k, 2) = q(i, j, k, 2) - Dfc(c, q(i, j, k, 1)) + tmp2 * ulap;
      }
}

void Operator(const Ctx& c, const FArr& q, const int* mx, double h, FArr& res) {
  if (c.ndims == 2) Operator2D(c, q, mx, h, res);
  else Operator3D(c, q, mx, h, res);
}

// Restriction2D/3D (gridutilities.f90:89-110, 406-433).  `a` is addressed
// with its own indices starting at 1 (the reference passes a(1:mx) sections).
void Restriction(const Ctx& c, const FArr& a, const int* mx, int nv, FArr& out) {
  int cm[3] = {mx[0] / 2, mx[1] / 2, c.ndims == 3 ? mx[2] / 2 : 1};
  out.alloc(1, cm[0], 1, cm[1], 1, cm[2], 1, nv);
  if (c.ndims == 2) {
    for (int v = 1; v <= nv; ++v)
      for (int jc = 1; jc <= cm[1]; ++jc)
        for (int ic = 1; ic <= cm[0]; ++ic) {
          int i = 2 * ic, j = 2 * jc;
          out(ic, jc, 1, v) = 0.25 * (a(i, j, 1, v) + a(i - 1, j, 1, v) + a(i, j - 1, 1, v) +
                                      a(i - 1, j - 1, 1, v));
        }
  } else {
    for (int v = 1; v <= nv; ++v)
      for (int kc = 1; kc <= cm[2]; ++kc)
        for (int jc = 1; jc <= cm[1]; ++jc)
          for (int ic = 1; ic <= cm[0]; ++ic) {
            int i = 2 * ic, j = 2 * jc, k = 2 * kc;
            out(ic, jc, kc, v) =
                0.125 * (a(i, j, k, v) + a(i - 1, j, k, v) + a(i, j - 1, k, v) +
                         a(i - 1, j - 1, k, v) + a(i, j, k - 1, v) + a(i - 1, j, k - 1, v) +
                         a(i, j - 1, k - 1, v) + a(i - 1, j - 1, k - 1, v));
          }
  }
}

// BiLinProlongationP1 / TriLinProlongationP1 (gridutilities.f90:137-175,
// 474-529).  a has bounds (0:cmx+1); out gets (0:mx+1) with mx = 2*cmx.
void ProlongationP1(const Ctx& c, const FArr& a, const int* cmx, int nv, FArr& out) {
  int mx0 = 2 * cmx[0], mx1 = 2 * cmx[1];
  if (c.ndims == 2) {
    FArr b;
    b.alloc(0, mx0 + 1, 0, cmx[1] + 1, 1, 1, 1, nv);
    for (int v = 1; v <= nv; ++v)
      for (int n = 0; n <= cmx[1] + 1; ++n)
        for (int m = 0; m <= cmx[0]; ++m) {
          b(2 * m, n, 1, v) = 3.0 * a(m, n, 1, v) + a(m + 1, n, 1, v);
          b(2 * m + 1, n, 1, v) = a(m, n, 1, v) + 3.0 * a(m + 1, n, 1, v);
        }
    out.alloc(0, mx0 + 1, 0, mx1 + 1, 1, 1, 1, nv);
    for (int v = 1; v <= nv; ++v)
      for (int n = 0; n <= cmx[1]; ++n)
        for (int i = 0; i <= mx0 + 1; ++i) {
          out(i, 2 * n, 1, v) = (3.0 * b(i, n, 1, v) + b(i, n + 1, 1, v)) / 16.0;
          out(i, 2 * n + 1, 1, v) = (b(i, n, 1, v) + 3.0 * b(i, n + 1, 1, v)) / 16.0;
        }
  } else {
    int mx2 = 2 * cmx[2];
    FArr b, cc;
    b.alloc(0, mx0 + 1, 0, cmx[1] + 1, 0, cmx[2] + 1, 1, nv);
    for (int v = 1; v <= nv; ++v)
      for (int p = 0; p <= cmx[2] + 1; ++p)
        for (int n = 0; n <= cmx[1] + 1; ++n)
          for (int m = 0; m <= cmx[0]; ++m) {
            b(2 * m, n, p, v) = 3.0 * a(m, n, p, v) + a(m + 1, n, p, v);
            b(2 * m + 1, n, p, v) = a(m, n, p, v) + 3.0 * a(m + 1, n, p, v);
          }
    cc.alloc(0, mx0 + 1, 0, mx1 + 1, 0, cmx[2] + 1, 1, nv);
    for (int v = 1; v <= nv; ++v)
      for (int p = 0; p <= cmx[2] + 1; ++p)
        for (int n = 0; n <= cmx[1]; ++n)
          for (int i = 0; i <= mx0 + 1; ++i) {
            cc(i, 2 * n, p, v) = 3.0 * b(i, n, p, v) + b(i, n + 1, p, v);
            cc(i, 2 * n + 1, p, v) = b(i, n, p, v) + 3.0 * b(i, n + 1, p, v);
          }
    out.alloc(0, mx0 + 1, 0, mx1 + 1, 0, mx2 + 1, 1, nv);
    for (int v = 1; v <= nv; ++v)
      for (int p = 0; p <= cmx[2]; ++p)
        for (int j = 0; j <= mx1 + 1; ++j)
          for (int i = 0; i <= mx0 + 1; ++i) {
            out(i, j, 2 * p, v) = (3.0 * cc(i, j, p, v) + cc(i, j, p + 1, v)) / 64.0;
            out(i, j, 2 * p + 1, v) = (cc(i, j, p, v) + 3.0 * cc(i, j, p + 1, v)) / 64.0;
          }
  }
}

// ---------------------------------------------------------------------------
// Physical boundary conditions: SetBC2D/SetBC3D (boundary.f90:643-891) with
// the problem module's UserBC2D/UserBC3D (problem.f90:646-756), mbc = 1.
// Returns nonzero for a code the reference stops on.
int SetBC2D(FArr& q, const int* mx, int nv, const int* mthbc) {
  const int ll = 0, ul1 = mx[0] + 1, ul2 = mx[1] + 1;
  for (int face = 1; face <= 4; ++face) {
    int code = mthbc[face - 1];
    if (code == 2 || code == 999) continue;
    if (code == 1) {
      for (int v = 1; v <= nv; ++v) {
        if (face == 1) for (int j = ll; j <= ul2; ++j) q(0, j, 1, v) = q(1, j, 1, v);
        if (face == 2) for (int j = ll; j <= ul2; ++j) q(mx[0] + 1, j, 1, v) = q(mx[0], j, 1, v);
        if (face == 3) for (int i = ll; i <= ul1; ++i) q(i, 0, 1, v) = q(i, 1, 1, v);
        if (face == 4) for (int i = ll; i <= ul1; ++i) q(i, mx[1] + 1, 1, v) = q(i, mx[1], 1, v);
      }
    } else if (code >= 10 && code <= 99) {
      // UserBC2D(q, ..., bcnow = face).
      if (face == 1)
        for (int v = 1; v <= nv; ++v)
          for (int j = ll; j <= ul2; ++j) q(0, j, 1, v) = 2.0 - q(1, j, 1, v);
      if (face == 2)
        for (int v = 1; v <= nv; ++v)
          for (int j = ll; j <= ul2; ++j) q(mx[0] + 1, j, 1, v) = 2.0 - q(mx[0], j, 1, v);
      if (face == 3)
        for (int v = 1; v <= 2; ++v)
          for (int i = ll; i <= ul1; ++i) q(i, 0, 1, v) = q(i, 1, 1, v);
      if (face == 4)
        for (int v = 1; v <= 2; ++v)
          for (int i = ll; i <= ul1; ++i) q(i, mx[1] + 1, 1, v) = q(i, mx[1], 1, v);
    } else {
      return -1;
    }
  }
  return 0;
}

int SetBC3D(FArr& q, const int* mx, int nv, const int* mthbc) {
  const int ll = 0, ul[3] = {mx[0] + 1, mx[1] + 1, mx[2] + 1};
  for (int face = 1; face <= 6; ++face) {
    int code = mthbc[face - 1];
    if (code == 2 || code == 999) continue;
    bool user = (code >= 10 && code <= 99);
    if (code != 1 && !user) return -1;
    int dim = (face - 1) / 2;
    bool hi = (face % 2) == 0;
    int g = hi ? mx[dim] + 1 : 0;   // ghost index along dim
    int s = hi ? mx[dim] : 1;       // source index along dim
    for (int v = 1; v <= nv; ++v)
      for (int k = ll; k <= ul[2]; ++k)
        for (int j = ll; j <= ul[1]; ++j)
          for (int i = ll; i <= ul[0]; ++i) {
            int idx[3] = {i, j, k};
            if (idx[dim] != g) continue;
            int src[3] = {i, j, k};
            src[dim] = s;
            double val = q(src[0], src[1], src[2], v);
            q(i, j, k, v) = user ? 2.0 - val : val;
          }
  }
  return 0;
}

int SetBC(const Ctx& c, Patch& p) {
  if (p.tobedeleted) return 0;
  if (c.ndims == 2) return SetBC2D(p.q, p.mx, p.nrvars, p.mthbc);
  return SetBC3D(p.q, p.mx, p.nrvars, p.mthbc);
}

// Coefficients of the Boundary module (boundary.f90:45-54).  Declared
// `real`; the reference builds with -fdefault-real-8 (makefile:85), so they
// are these FP64 quotients.
constexpr double kA1 = -(1.0 / 5.0), kA2 = 2.0 / 3.0, kA3 = 8.0 / 15.0;
constexpr double kB1 = 5.0 / 32.0, kB2 = 15.0 / 16.0, kB3 = -(3.0 / 32.0);

// Interpolate2D (boundary.f90:135-323), mbc = 1: ghosts of a fine patch on
// its internal faces (codes 2 and 999) from two fine cells and one coarse
// value along a diagonal; ipass 1 = red, 2 = black, 0 = both.  Corners are
// set whatever the face codes are (SetBC overwrites the physical ones).
// Every statement reads interior fine cells and coarse cells only.
void Interpolate2D(FArr& qf, const FArr& qc, const int* mx, int nv, const int mb[3][2],
                   const int* mthbc, int ipass) {
  const int m1 = mx[0], m2 = mx[1];
  const int b11 = mb[0][0], b12 = mb[0][1], b21 = mb[1][0], b22 = mb[1][1];
  const bool red = ipass == 1 || ipass == 0, black = ipass == 2 || ipass == 0;
  auto Q = [&](int i, int j, int v) -> double& { return qf(i, j, 1, v); };
  auto C = [&](int i, int j, int v) { return qc(i, j, 1, v); };
  for (int v = 1; v <= nv; ++v) {
    // Corners (boundary.f90:147-172).
    if (red) {
      Q(m1 + 1, m2 + 1, v) = kA1 * Q(m1 - 1, m2 - 1, v) + kA2 * Q(m1, m2, v) +
                             kA3 * C(b12 + 1, b22 + 1, v);
      Q(0, 0, v) = kA1 * Q(2, 2, v) + kA2 * Q(1, 1, v) + kA3 * C(b11 - 1, b21 - 1, v);
    }
    if (black) {
      Q(m1 + 1, 0, v) = kA1 * Q(m1 - 1, 2, v) + kA2 * Q(m1, 1, v) + kA3 * C(b12 + 1, b21 - 1, v);
      Q(0, m2 + 1, v) = kA1 * Q(2, m2 - 1, v) + kA2 * Q(1, m2, v) + kA3 * C(b11 - 1, b22 + 1, v);
    }
  }
  auto internal = [](int code) { return code == 2 || code == 999; };
  // A face's interior ghosts: the regular section of one colour plus the end
  // ghost whose coarse value is the three-point fit (b1, b2, b3) along the
  // face.  t counts the elements of the array section.
  for (int v = 1; v <= nv; ++v) {
    if (internal(mthbc[0])) {  // face 1 (boundary.f90:176-212)
      if (red) {
        for (int t = 0; 2 + 2 * t <= m2 - 2; ++t) {
          const int j = 2 + 2 * t;
          Q(0, j, v) = kA1 * Q(2, 4 + 2 * t, v) + kA2 * Q(1, 3 + 2 * t, v) +
                       kA3 * C(b11 - 1, b21 + t, v);
        }
        Q(0, m2, v) = kA1 * Q(2, m2, v) + kA2 * Q(1, m2, v) +
                      kA3 * (kB1 * C(b11 - 1, b22 + 1, v) + kB2 * C(b11 - 1, b22, v) +
                             kB3 * C(b11 - 1, b22 - 1, v));
      }
      if (black) {
        for (int t = 0; 3 + 2 * t <= m2 - 1; ++t) {
          const int j = 3 + 2 * t;
          Q(0, j, v) = kA1 * Q(2, 1 + 2 * t, v) + kA2 * Q(1, 2 + 2 * t, v) +
                       kA3 * C(b11 - 1, b21 + 1 + t, v);
        }
        Q(0, 1, v) = kA1 * Q(2, 1, v) + kA2 * Q(1, 1, v) +
                     kA3 * (kB1 * C(b11 - 1, b21 - 1, v) + kB2 * C(b11 - 1, b21, v) +
                            kB3 * C(b11 - 1, b21 + 1, v));
      }
    }
    if (internal(mthbc[1])) {  // face 2 (boundary.f90:214-250)
      if (red) {
        for (int t = 0; 3 + 2 * t <= m2 - 1; ++t) {
          const int j = 3 + 2 * t;
          Q(m1 + 1, j, v) = kA1 * Q(m1 - 1, 1 + 2 * t, v) + kA2 * Q(m1, 2 + 2 * t, v) +
                            kA3 * C(b12 + 1, b21 + 1 + t, v);
        }
        Q(m1 + 1, 1, v) = kA1 * Q(m1 - 1, 1, v) + kA2 * Q(m1, 1, v) +
                          kA3 * (kB1 * C(b12 + 1, b21 - 1, v) + kB2 * C(b12 + 1, b21, v) +
                                 kB3 * C(b12 + 1, b21 + 1, v));
      }
      if (black) {
        for (int t = 0; 2 + 2 * t <= m2 - 2; ++t) {
          const int j = 2 + 2 * t;
          Q(m1 + 1, j, v) = kA1 * Q(m1 - 1, 4 + 2 * t, v) + kA2 * Q(m1, 3 + 2 * t, v) +
                            kA3 * C(b12 + 1, b21 + t, v);
        }
        Q(m1 + 1, m2, v) = kA1 * Q(m1 - 1, m2, v) + kA2 * Q(m1, m2, v) +
                           kA3 * (kB1 * C(b12 + 1, b22 + 1, v) + kB2 * C(b12 + 1, b22, v) +
                                  kB3 * C(b12 + 1, b22 - 1, v));
      }
    }
    if (internal(mthbc[2])) {  // face 3 (boundary.f90:252-287)
      if (red) {
        for (int t = 0; 2 + 2 * t <= m1 - 2; ++t) {
          const int i = 2 + 2 * t;
          Q(i, 0, v) = kA1 * Q(4 + 2 * t, 2, v) + kA2 * Q(3 + 2 * t, 1, v) +
                       kA3 * C(b11 + t, b21 - 1, v);
        }
        Q(m1, 0, v) = kA1 * Q(m1, 2, v) + kA2 * Q(m1, 1, v) +
                      kA3 * (kB1 * C(b12 + 1, b21 - 1, v) + kB2 * C(b12, b21 - 1, v) +
                             kB3 * C(b12 - 1, b21 - 1, v));
      }
      if (black) {
        for (int t = 0; 3 + 2 * t <= m1 - 1; ++t) {
          const int i = 3 + 2 * t;
          Q(i, 0, v) = kA1 * Q(1 + 2 * t, 2, v) + kA2 * Q(2 + 2 * t, 1, v) +
                       kA3 * C(b11 + 1 + t, b21 - 1, v);
        }
        Q(1, 0, v) = kA1 * Q(1, 2, v) + kA2 * Q(1, 1, v) +
                     kA3 * (kB1 * C(b11 - 1, b21 - 1, v) + kB2 * C(b11, b21 - 1, v) +
                            kB3 * C(b11 + 1, b21 - 1, v));
      }
    }
    if (internal(mthbc[3])) {  // face 4 (boundary.f90:289-321)
      if (red) {
        for (int t = 0; 3 + 2 * t <= m1 - 1; ++t) {
          const int i = 3 + 2 * t;
          Q(i, m2 + 1, v) = kA1 * Q(1 + 2 * t, m2 - 1, v) + kA2 * Q(2 + 2 * t, m2, v) +
                            kA3 * C(b11 + 1 + t, b22 + 1, v);
        }
        Q(1, m2 + 1, v) = kA1 * Q(1, m2 - 1, v) + kA2 * Q(1, m2, v) +
                          kA3 * (kB1 * C(b11 - 1, b22 + 1, v) + kB2 * C(b11, b22 + 1, v) +
                                 kB3 * C(b11 + 1, b22 + 1, v));
      }
      if (black) {
        for (int t = 0; 2 + 2 * t <= m1 - 2; ++t) {
          const int i = 2 + 2 * t;
          Q(i, m2 + 1, v) = kA1 * Q(4 + 2 * t, m2 - 1, v) + kA2 * Q(3 + 2 * t, m2, v) +
                            kA3 * C(b11 + t, b22 + 1, v);
        }
        Q(m1, m2 + 1, v) = kA1 * Q(m1, m2 - 1, v) + kA2 * Q(m1, m2, v) +
                           kA3 * (kB1 * C(b12 + 1, b22 + 1, v) + kB2 * C(b12, b22 + 1, v) +
                                  kB3 * C(b12 - 1, b22 + 1, v));
      }
    }
  }
}

constexpr double kC1 = 9.0 / 16.0, kC2 = 3.0 / 16.0, kC3 = 3.0 / 16.0, kC4 = 1.0 / 16.0;

// GetFaceIndex (boundary.f90:1271-1297) of dimension d (0-based): the ghost,
// second and first interior fine indices, the parent's index outside the
// patch's footprint and the parent's boundary index of the footprint.
struct FaceIdx {
  int g, s, f, p, b;
};
FaceIdx GetFaceIndex(const int* mx, const int mb[3][2], int d, int parity) {
  if (parity == 1) return {0, 2, 1, mb[d][0] - 1, mb[d][0]};
  return {mx[d] + 1, mx[d] - 1, mx[d], mb[d][1] + 1, mb[d][1]};
}

// One dimension of an Interpolate3D array statement: the n elements of the
// target section, of the two fine sources (a1 and a2 terms) and of the
// parent section advance together, the fine indices by df, the parent's by dc.
struct Ax {
  int t, s, f, c, n, df, dc;
};
Ax ax_fixed(const FaceIdx& F) { return {F.g, F.s, F.f, F.p, 1, 0, 0}; }
// The same fine index i in target and sources (the parent index along this
// dimension is given by the statement's parent combination).
Ax ax_at(int i) { return {i, i, i, 0, 1, 0, 0}; }
// Target 3:m-1:2, sources 1:m-3:2 and 2:m-2:2, parent lo+1:...
Ax ax_odd(int m, int lo) { return {3, 1, 2, lo + 1, m >= 4 ? (m - 2) / 2 : 0, 2, 1}; }
// Target 2:m-2:2, sources 4:m:2 and 3:m-1:2, parent lo:...
Ax ax_even(int m, int lo) { return {2, 4, 3, lo, m >= 4 ? (m - 2) / 2 : 0, 2, 1}; }

// The parent term of a statement: one parent value (kind 0); the three-point
// fit b1, b2, b3 over indices k[0..2] along dimension d (kind 1); the
// four-point corner fit c1..c4 over (k[0], k[1]) along d and (k2[0], k2[1])
// along d2 (kind 2: c1 at (k[0], k2[0]), c2 at (k[1], k2[0]), c3 at
// (k[0], k2[1]), c4 at (k[1], k2[1])).
struct Par {
  int kind, d, k[3], d2, k2[2];
};
Par par_one() { return {0, 0, {0, 0, 0}, 0, {0, 0}}; }
Par par_fit(int d, int k0, int k1, int k2) { return {1, d, {k0, k1, k2}, 0, {0, 0}}; }
Par par_corner(int d, int f5, int f4, int d2, int g5, int g4) {
  return {2, d, {f5, f4, 0}, d2, {g5, g4}};
}

// qf(target) = a1*qf(second) + a2*qf(first) + a3*parent, elementwise; the
// right-hand side reads interior fine cells and parent cells only.
void stmt3(FArr& qf, const FArr& qc, int nv, const Ax& X, const Ax& Y, const Ax& Z,
           const Par& P) {
  const Ax A[3] = {X, Y, Z};
  for (int v = 1; v <= nv; ++v)
    for (int c = 0; c < Z.n; ++c)
      for (int b = 0; b < Y.n; ++b)
        for (int a = 0; a < X.n; ++a) {
          const int e[3] = {a, b, c};
          int T[3], S[3], F[3], C[3];
          for (int d = 0; d < 3; ++d) {
            T[d] = A[d].t + e[d] * A[d].df;
            S[d] = A[d].s + e[d] * A[d].df;
            F[d] = A[d].f + e[d] * A[d].df;
            C[d] = A[d].c + e[d] * A[d].dc;
          }
          auto pc = [&](int d, int k, int d2, int k2) {
            int I[3] = {C[0], C[1], C[2]};
            I[d] = k;
            if (d2 >= 0) I[d2] = k2;
            return qc(I[0], I[1], I[2], v);
          };
          double par;
          if (P.kind == 0)
            par = qc(C[0], C[1], C[2], v);
          else if (P.kind == 1)
            par = kB1 * pc(P.d, P.k[0], -1, 0) + kB2 * pc(P.d, P.k[1], -1, 0) +
                  kB3 * pc(P.d, P.k[2], -1, 0);
          else
            par = kC1 * pc(P.d, P.k[0], P.d2, P.k2[0]) + kC2 * pc(P.d, P.k[1], P.d2, P.k2[0]) +
                  kC3 * pc(P.d, P.k[0], P.d2, P.k2[1]) + kC4 * pc(P.d, P.k[1], P.d2, P.k2[1]);
          qf(T[0], T[1], T[2], v) =
              kA1 * qf(S[0], S[1], S[2], v) + kA2 * qf(F[0], F[1], F[2], v) + kA3 * par;
        }
}

// Interpolate3D (boundary.f90:1299-1799), mbc = 1, statement by statement:
// (1) the 8 corners, (2) the 12 edges, (3) the 6 faces (internal faces only)
// with their corner cells.  Corners and edges on a physical face are skipped
// only in the red pass (ipass = 1).  The check for edges 1-4 tests the z
// face code against 99, not 999 (boundary.f90:1354), and is kept.  Every
// statement reads interior fine cells and parent cells only.
void Interpolate3D(FArr& qf, const FArr& qc, const int* mx, int nv, const int mb[3][2],
                   const int* mthbc, int ipass) {
  auto internal = [](int code) { return code == 2 || code == 999; };
  auto skip = [&](int face, bool typo) {
    const int code = mthbc[face];
    const bool keep = typo ? (code == 2 || code == 99) : internal(code);
    return !keep && ipass == 1;
  };
  // (1) Corners (boundary.f90:1322-1342).
  for (int p1 = 1; p1 <= 2; ++p1) {
    if (skip(p1 - 1, false)) continue;
    const FaceIdx F1 = GetFaceIndex(mx, mb, 0, p1);
    for (int p2 = 1; p2 <= 2; ++p2) {
      if (skip(p2 + 1, false)) continue;
      const FaceIdx F2 = GetFaceIndex(mx, mb, 1, p2);
      for (int p3 = 1; p3 <= 2; ++p3) {
        if (skip(p3 + 3, false)) continue;
        const FaceIdx F3 = GetFaceIndex(mx, mb, 2, p3);
        stmt3(qf, qc, nv, ax_fixed(F1), ax_fixed(F2), ax_fixed(F3), par_one());
      }
    }
  }
  // (2) Edges, along the dimension `e` not fixed (boundary.f90:1344-1478):
  // odd cells from the diagonal below, the first cell with the fit at the
  // footprint's low end, even cells from the diagonal above, the last cell
  // with the fit at the high end.
  auto edge = [&](int e, const Ax& A, const Ax& B) {
    const int m = mx[e], lo = mb[e][0], hi = mb[e][1];
    auto put = [&](const Ax& L, const Par& P) {
      Ax D[3];
      int k = 0;
      for (int d = 0; d < 3; ++d) D[d] = d == e ? L : (k++ == 0 ? A : B);
      stmt3(qf, qc, nv, D[0], D[1], D[2], P);
    };
    put(ax_odd(m, lo), par_one());
    put(ax_at(1), par_fit(e, lo - 1, lo, lo + 1));
    put(ax_even(m, lo), par_one());
    put(ax_at(m), par_fit(e, hi + 1, hi, hi - 1));
  };
  for (int p1 = 1; p1 <= 2; ++p1) {  // edges 1-4: dimensions 1 and 3 fixed
    if (skip(p1 - 1, false)) continue;
    const FaceIdx F1 = GetFaceIndex(mx, mb, 0, p1);
    for (int p3 = 1; p3 <= 2; ++p3) {
      if (skip(p3 + 3, true)) continue;
      const FaceIdx F3 = GetFaceIndex(mx, mb, 2, p3);
      edge(1, ax_fixed(F1), ax_fixed(F3));
    }
  }
  for (int p1 = 1; p1 <= 2; ++p1) {  // edges 5-8: dimensions 1 and 2 fixed
    if (skip(p1 - 1, false)) continue;
    const FaceIdx F1 = GetFaceIndex(mx, mb, 0, p1);
    for (int p2 = 1; p2 <= 2; ++p2) {
      if (skip(p2 + 1, false)) continue;
      const FaceIdx F2 = GetFaceIndex(mx, mb, 1, p2);
      edge(2, ax_fixed(F1), ax_fixed(F2));
    }
  }
  for (int p2 = 1; p2 <= 2; ++p2) {  // edges 9-12: dimensions 2 and 3 fixed
    if (skip(p2 + 1, false)) continue;
    const FaceIdx F2 = GetFaceIndex(mx, mb, 1, p2);
    for (int p3 = 1; p3 <= 2; ++p3) {
      if (skip(p3 + 3, false)) continue;
      const FaceIdx F3 = GetFaceIndex(mx, mb, 2, p3);
      edge(0, ax_fixed(F2), ax_fixed(F3));
    }
  }
  // (3) Faces (boundary.f90:1480-1797), internal faces only.  On face
  // dimension d with the other dimensions u < w: yellow (even, even) and blue
  // (odd, odd) cells in one colour, green (odd, even) and red (even, odd) in
  // the other, each as the interior section plus the strips next to the
  // face's edges; then its four corner cells with the four-point fit.  (Faces
  // 3 and 4 list the strips of green and red the other way round; the strips
  // are disjoint and in the same colour, so the result is the same.)
  for (int d = 0; d < 3; ++d) {
    const int u = d == 0 ? 1 : 0, w = d == 2 ? 1 : 2;
    const int mu = mx[u], mw = mx[w];
    const int u1 = mb[u][0], u2 = mb[u][1], w1 = mb[w][0], w2 = mb[w][1];
    for (int p = 1; p <= 2; ++p) {
      if (!internal(mthbc[2 * d + p - 1])) continue;
      const FaceIdx F = GetFaceIndex(mx, mb, d, p);
      auto put = [&](const Ax& U, const Ax& W, const Par& P) {
        Ax D[3];
        D[d] = ax_fixed(F);
        D[u] = U;
        D[w] = W;
        stmt3(qf, qc, nv, D[0], D[1], D[2], P);
      };
      if (ipass == 0 || (p + ipass) % 2 == 0) {
        // Yellow.
        put(ax_even(mu, u1), ax_even(mw, w1), par_one());
        put(ax_at(mu), ax_even(mw, w1), par_fit(u, u2 + 1, u2, u2 - 1));
        put(ax_even(mu, u1), ax_at(mw), par_fit(w, w2 + 1, w2, w2 - 1));
        // Blue.
        put(ax_odd(mu, u1), ax_odd(mw, w1), par_one());
        put(ax_odd(mu, u1), ax_at(1), par_fit(w, w1 - 1, w1, w1 + 1));
        put(ax_at(1), ax_odd(mw, w1), par_fit(u, u1 - 1, u1, u1 + 1));
      }
      if (ipass == 0 || (p + ipass) % 2 == 1) {
        // Green.
        put(ax_odd(mu, u1), ax_even(mw, w1), par_one());
        put(ax_at(1), ax_even(mw, w1), par_fit(u, u1 - 1, u1, u1 + 1));
        put(ax_odd(mu, u1), ax_at(mw), par_fit(w, w2 + 1, w2, w2 - 1));
        // Red.
        put(ax_even(mu, u1), ax_odd(mw, w1), par_one());
        put(ax_even(mu, u1), ax_at(1), par_fit(w, w1 - 1, w1, w1 + 1));
        put(ax_at(mu), ax_odd(mw, w1), par_fit(u, u2 + 1, u2, u2 - 1));
      }
      // Corner cells of the face.
      for (int pu = 1; pu <= 2; ++pu) {
        const FaceIdx Fu = GetFaceIndex(mx, mb, u, pu);
        for (int pw = 1; pw <= 2; ++pw) {
          const FaceIdx Fw = GetFaceIndex(mx, mb, w, pw);
          put(ax_at(Fu.f), ax_at(Fw.f), par_corner(u, Fu.b, Fu.p, w, Fw.b, Fw.p));
        }
      }
    }
  }
}

// GhostOverlap (boundary.f90:346-415), mbc = 1: each grid's ghost ring takes
// the other grid's interior values where they overlap (corners included).
void GhostOverlap(const Ctx& c, Patch& g1, Patch& g2) {
  const int mbc = g2.mbc, nv = g1.nrvars, nd = c.ndims;
  int mg1[3][2], mg2[3][2], ovg[3][2], ovg1[3][2], ovg2[3][2];
  for (int n = 0; n < 3; ++n)
    for (int s = 0; s < 2; ++s) {
      mg1[n][s] = n < nd ? g1.mglobal[n][s] : 1;
      mg2[n][s] = n < nd ? g2.mglobal[n][s] : 1;
      ovg[n][s] = ovg1[n][s] = ovg2[n][s] = 1;
    }
  for (int n = 0; n < nd; ++n) {
    ovg[n][0] = std::max(mg1[n][0] - mbc, mg2[n][0] - mbc);
    ovg[n][1] = std::min(mg1[n][1] + mbc, mg2[n][1] + mbc);
  }
  for (int n = 0; n < nd; ++n)
    if (ovg[n][1] - ovg[n][0] < 0) return;
  for (int n = 0; n < nd; ++n) {
    ovg1[n][0] = std::max(ovg[n][0], mg2[n][0]);
    ovg1[n][1] = std::min(ovg[n][1], mg2[n][1]);
    ovg2[n][0] = std::max(ovg[n][0], mg1[n][0]);
    ovg2[n][1] = std::min(ovg[n][1], mg1[n][1]);
  }
  // grid1(ovg1 - mg1 + 1) = grid2(ovg1 - mg2 + 1), then the other way.
  auto copy = [&](Patch& dst, const int (*mgd)[2], const Patch& src, const int (*mgs)[2],
                  const int (*box)[2]) {
    const int k0 = nd == 3 ? box[2][0] : 1, k1 = nd == 3 ? box[2][1] : 1;
    for (int v = 1; v <= nv; ++v)
      for (int k = k0; k <= k1; ++k)
        for (int j = box[1][0]; j <= box[1][1]; ++j)
          for (int i = box[0][0]; i <= box[0][1]; ++i) {
            const int dk = nd == 3 ? k - mgd[2][0] + 1 : 1, sk = nd == 3 ? k - mgs[2][0] + 1 : 1;
            dst.q(i - mgd[0][0] + 1, j - mgd[1][0] + 1, dk, v) =
                src.q(i - mgs[0][0] + 1, j - mgs[1][0] + 1, sk, v);
          }
  };
  // The transfers read interior cells only, so element order is immaterial.
  copy(g1, mg1, g2, mg2, ovg1);
  copy(g2, mg2, g1, mg1, ovg2);
}

// PeriodicBC (boundary.f90:417-483), mbc = 1 and qpo = 0: a grid whose two
// faces of a dimension are periodic copies its first interior layer into the
// high ghost layer, then its last into the low one, dimension by dimension,
// whole layers (the ghost rows of the other dimensions included).
void PeriodicBC(const Ctx& c, Patch& p) {
  if (p.tobedeleted) return;
  const int nd = c.ndims;
  const int lo[3] = {0, 0, nd == 3 ? 0 : 1};
  const int hi[3] = {p.mx[0] + 1, p.mx[1] + 1, nd == 3 ? p.mx[2] + 1 : 1};
  for (int dim = 0; dim < nd; ++dim) {
    if (!(p.mthbc[2 * dim] == 2 && p.mthbc[2 * dim + 1] == 2)) continue;
    const int m = p.mx[dim];
    for (int v = 1; v <= p.nrvars; ++v)
      for (int pass = 0; pass < 2; ++pass) {
        const int g = pass == 0 ? m + 1 : 0, from = pass == 0 ? 1 : m;
        for (int k = lo[2]; k <= hi[2]; ++k)
          for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
              int idx[3] = {i, j, k};
              if (idx[dim] != g) continue;
              int src[3] = {i, j, k};
              src[dim] = from;
              p.q(i, j, k, v) = p.q(src[0], src[1], src[2], v);
            }
      }
  }
}

// SetGhost (boundary.f90:58-89): above the root level, coarse-fine
// interpolation on every grid (ApplyOnLevel order), then the sibling
// exchange over all pairs (ApplyOnLevelPairs: each grid with every later
// one); with periodic faces, PeriodicBC on every grid (periodic grids exist
// at and below the root only: TransferPeriodicBC between refined grids is
// not restated); then the physical boundary conditions.
int SetGhost(Ctx& c, int level, int ipass) {
  int err = 0;
  if (level > Ctx::rootlevel) {
    std::vector<Patch*>& L = c.on(level);
    for (Patch* p : L) {
      if (p->tobedeleted) continue;
      if (c.ndims == 2)
        Interpolate2D(p->q, p->parent->q, p->mx, p->nrvars, p->mbounds, p->mthbc, ipass);
      else
        Interpolate3D(p->q, p->parent->q, p->mx, p->nrvars, p->mbounds, p->mthbc, ipass);
    }
    for (size_t a = 0; a < L.size(); ++a)
      for (size_t b = a + 1; b < L.size(); ++b)
        if (!L[a]->tobedeleted && !L[b]->tobedeleted) GhostOverlap(c, *L[a], *L[b]);
  }
  if (c.periodic)
    for (Patch* p : c.on(level)) PeriodicBC(c, *p);
  for (Patch* p : c.on(level)) err |= SetBC(c, *p);
  return err;
}

// GetCoarseGhostPoints (boundary.f90:1203-1269).
void GetCoarseGhostPoints(const Ctx& c, Patch& p) {
  if (p.tobedeleted) return;
  Patch& par = *p.parent;
  int nv = p.nrvars;
  int cmx[3] = {1, 1, 1}, il[3] = {1, 1, 1}, ih[3] = {1, 1, 1}, jl[3] = {1, 1, 1},
      jh[3] = {1, 1, 1}, mb[3][2] = {{1, 1}, {1, 1}, {1, 1}};
  for (int n = 0; n < c.ndims; ++n) {
    cmx[n] = p.mx[n] / 2;
    il[n] = 0;
    ih[n] = cmx[n] + 1;
    mb[n][0] = p.mbounds[n][0];
    mb[n][1] = p.mbounds[n][1];
    jl[n] = mb[n][0] - 1;
    jh[n] = mb[n][1] + 1;
  }
  for (int v = 1; v <= nv; ++v) {
    // Faces 1 and 2.
    for (int k = il[2], pk = jl[2]; k <= ih[2]; ++k, ++pk)
      for (int j = il[1], pj = jl[1]; j <= ih[1]; ++j, ++pj) {
        p.qc(il[0], j, k, v) = par.q(jl[0], pj, pk, v);
        p.qc(ih[0], j, k, v) = par.q(jh[0], pj, pk, v);
      }
    // Faces 3 and 4.
    for (int k = il[2], pk = jl[2]; k <= ih[2]; ++k, ++pk)
      for (int i = 1, pi = mb[0][0]; i <= cmx[0]; ++i, ++pi) {
        p.qc(i, il[1], k, v) = par.q(pi, jl[1], pk, v);
        p.qc(i, ih[1], k, v) = par.q(pi, jh[1], pk, v);
      }
    if (c.ndims == 3) {
      for (int j = 1, pj = mb[1][0]; j <= cmx[1]; ++j, ++pj)
        for (int i = 1, pi = mb[0][0]; i <= cmx[0]; ++i, ++pi) {
          p.qc(i, j, il[2], v) = par.q(pi, pj, jl[2], v);
          p.qc(i, j, ih[2], v) = par.q(pi, pj, jh[2], v);
        }
    }
  }
}

// ---------------------------------------------------------------------------
// AFAS routines (lib/afasroutines.f90).
inline int cmx_of(const Ctx& c, const Patch& p, int n) {
  return n < c.ndims ? p.mx[n] / 2 : 1;
}

// Residual (afas:799-840): rf = f - Operator(q).
void Residual(const Ctx& c, Patch& p) {
  FArr res;
  Operator(c, p.q, p.mx, p.dx[0], res);
  int n3 = c.ndims == 3 ? p.mx[2] : 1;
  for (int v = 1; v <= p.nrvars; ++v)
    for (int k = 1; k <= n3; ++k)
      for (int j = 1; j <= p.mx[1]; ++j)
        for (int i = 1; i <= p.mx[0]; ++i) p.rf(i, j, k, v) = p.f(i, j, k, v) - res(i, j, k, v);
}

// SquareSum (afas:210-221): sum(rf*rf), sequential, column-major.
double SquareSum(const Ctx& c, const Patch& p) {
  double s = 0.0;
  int n3 = c.ndims == 3 ? p.mx[2] : 1;
  for (int v = 1; v <= p.nrvars; ++v)
    for (int k = 1; k <= n3; ++k)
      for (int j = 1; j <= p.mx[1]; ++j)
        for (int i = 1; i <= p.mx[0]; ++i) {
          double r = p.rf(i, j, k, v);
          s = s + r * r;
        }
  return s;
}

// ErrorAFAS with errortype 1 + L2Error (afas:108-179).
double ErrorAFAS(Ctx& c, int level) {
  double ir1 = 0.0, ir2 = 0.0;
  for (Patch* p : c.on(level)) {
    Residual(c, *p);
    ir1 = SquareSum(c, *p) + ir1;
    long ncell = 1;
    for (int n = 0; n < c.ndims; ++n) ncell *= p->mx[n];
    ir2 = (double)(p->nrvars * ncell) + ir2;
  }
  return std::sqrt(ir1 / ir2);
}

// Copy a (1:cmx) restriction result into parent(mb) -- shared by
// FillDownLevel and RestrictSolution.
void StoreIntoParent(const Ctx& c, const FArr& src, FArr& dst, const Patch& p, int nv) {
  int cm[3] = {cmx_of(c, p, 0), cmx_of(c, p, 1), cmx_of(c, p, 2)};
  int mb0[3] = {p.mbounds[0][0], p.mbounds[1][0], c.ndims == 3 ? p.mbounds[2][0] : 1};
  for (int v = 1; v <= nv; ++v)
    for (int k = 1; k <= cm[2]; ++k)
      for (int j = 1; j <= cm[1]; ++j)
        for (int i = 1; i <= cm[0]; ++i)
          dst(mb0[0] + i - 1, mb0[1] + j - 1, mb0[2] + k - 1, v) = src(i, j, k, v);
}

// FillDownLevel (afas:241-310).
void FillDownLevel(Ctx& c, Patch& p, bool source) {
  if (p.tobedeleted) return;
  FArr r;
  if (source) {
    Restriction(c, p.f, p.mx, p.nrvars, r);
    StoreIntoParent(c, r, p.parent->f, p, p.nrvars);
  } else {
    Restriction(c, p.q, p.mx, p.nrvars, r);
    StoreIntoParent(c, r, p.parent->q, p, p.nrvars);
  }
}

// FillDown (afas:223-239).
void FillDown(Ctx& c, bool source) {
  for (int level = c.finestlevel; level >= c.minlevel + 1; --level) {
    for (Patch* p : c.on(level)) FillDownLevel(c, *p, source);
    if (!source) SetGhost(c, level - 1, 0);
  }
}

// GetSourceFunction (afas:312-367): ftmp = Source(q, qold).
void GetSourceFunction(Ctx& c, Patch& p) {
  if (p.tobedeleted) return;
  int n3 = c.ndims == 3 ? p.mx[2] : 1;
  for (int k = 1; k <= n3; ++k)
    for (int j = 1; j <= p.mx[1]; ++j)
      for (int i = 1; i <= p.mx[0]; ++i) p.ftmp(i, j, k, 1) = p.qold(i, j, k, 1);
  for (int k = 1; k <= n3; ++k)
    for (int j = 1; j <= p.mx[1]; ++j)
      for (int i = 1; i <= p.mx[0]; ++i) p.ftmp(i, j, k, 2) = -Dfe(c, p.qold(i, j, k, 1));
}

// UpdateSourceFunction (afas:427-486): f = ftmp + SourceUpdate (= 0).
void UpdateSourceFunction(Ctx& c, Patch& p) {
  if (p.tobedeleted) return;
  int n3 = c.ndims == 3 ? p.mx[2] : 1;
  for (int v = 1; v <= p.nrvars; ++v)
    for (int k = 1; k <= n3; ++k)
      for (int j = 1; j <= p.mx[1]; ++j)
        for (int i = 1; i <= p.mx[0]; ++i) p.f(i, j, k, v) = p.ftmp(i, j, k, v) + 0.0;
}

// RelaxPatch (afas:549-598).
void RelaxPatch(Ctx& c, Patch& p, int ipass) {
  if (p.tobedeleted) return;
  if (c.ndims == 2) RelaxGrid2D(c, p.q, p.f, p.mx, p.dx[0], ipass);
  else RelaxGrid3D(c, p.q, p.f, p.mx, p.dx[0], ipass);
}

// LevelRelax (afas:523-547).
void LevelRelax(Ctx& c, int level) {
  for (int pass = 1; pass <= c.nsmoothingpasses; ++pass)
    for (int rb = 1; rb <= 2; ++rb) {
      for (Patch* p : c.on(level)) RelaxPatch(c, *p, rb);
      SetGhost(c, level, rb);
    }
}

// RestrictSolution (afas:600-644).
void RestrictSolution(Ctx& c, Patch& p) {
  if (p.tobedeleted) return;
  FArr r;
  Restriction(c, p.q, p.mx, p.nrvars, r);
  int cm[3] = {cmx_of(c, p, 0), cmx_of(c, p, 1), cmx_of(c, p, 2)};
  for (int v = 1; v <= p.nrvars; ++v)
    for (int k = 1; k <= cm[2]; ++k)
      for (int j = 1; j <= cm[1]; ++j)
        for (int i = 1; i <= cm[0]; ++i) p.qc(i, j, k, v) = r(i, j, k, v);
  StoreIntoParent(c, p.qc, p.parent->q, p, p.nrvars);
}

// CoarseLoadingFunction (afas:646-714):
//   parent%f(mb) = Restriction(rf) + Operator(qc incl. ring, h = parent%dx).
void CoarseLoadingFunction(Ctx& c, Patch& p) {
  if (p.tobedeleted) return;
  Patch& par = *p.parent;
  Residual(c, p);
  FArr r, op;
  Restriction(c, p.rf, p.mx, p.nrvars, r);
  int cm[3] = {cmx_of(c, p, 0), cmx_of(c, p, 1), cmx_of(c, p, 2)};
  Operator(c, p.qc, cm, par.dx[0], op);
  FArr sum;
  sum.alloc(1, cm[0], 1, cm[1], 1, cm[2], 1, p.nrvars);
  for (int v = 1; v <= p.nrvars; ++v)
    for (int k = 1; k <= cm[2]; ++k)
      for (int j = 1; j <= cm[1]; ++j)
        for (int i = 1; i <= cm[0]; ++i) sum(i, j, k, v) = r(i, j, k, v) + op(i, j, k, v);
  StoreIntoParent(c, sum, par.f, p, p.nrvars);
}

// CorrectFine with mbc = 1 (afas:842-963).
void CorrectFine(Ctx& c, Patch& p) {
  if (p.tobedeleted) return;
  Patch& par = *p.parent;
  int cm[3] = {cmx_of(c, p, 0), cmx_of(c, p, 1), cmx_of(c, p, 2)};
  int nv = p.nrvars;
  int lo3 = c.ndims == 3 ? 0 : 1, hi3 = c.ndims == 3 ? cm[2] + 1 : 1;
  int off[3] = {p.mbounds[0][0] - 1, p.mbounds[1][0] - 1,
                c.ndims == 3 ? p.mbounds[2][0] - 1 : 0};
  // qc(0:cmx+1) = parent%q(mb-1:mb+1) - qc(0:cmx+1)
  for (int v = 1; v <= nv; ++v)
    for (int k = lo3; k <= hi3; ++k)
      for (int j = 0; j <= cm[1] + 1; ++j)
        for (int i = 0; i <= cm[0] + 1; ++i)
          p.qc(i, j, k, v) = par.q(off[0] + i, off[1] + j, c.ndims == 3 ? off[2] + k : 1, v) -
                             p.qc(i, j, k, v);
  FArr pr;
  ProlongationP1(c, p.qc, cm, nv, pr);
  int mlo3 = c.ndims == 3 ? 0 : 1, mhi3 = c.ndims == 3 ? p.mx[2] + 1 : 1;
  for (int v = 1; v <= nv; ++v)
    for (int k = mlo3; k <= mhi3; ++k)
      for (int j = 0; j <= p.mx[1] + 1; ++j)
        for (int i = 0; i <= p.mx[0] + 1; ++i) p.q(i, j, k, v) = p.q(i, j, k, v) + pr(i, j, k, v);
}

// AFASVcycle (afas:488-521).
void AFASVcycle(Ctx& c, int level) {
  LevelRelax(c, level);
  if (level > c.minlevel) {
    for (Patch* p : c.on(level)) RestrictSolution(c, *p);
    SetGhost(c, level - 1, 0);
    for (Patch* p : c.on(level)) GetCoarseGhostPoints(c, *p);
    for (Patch* p : c.on(level)) CoarseLoadingFunction(c, *p);
    AFASVcycle(c, level - 1);
    for (Patch* p : c.on(level)) CorrectFine(c, *p);
    SetGhost(c, level, 0);
    LevelRelax(c, level);
  }
}

// MultigridIterations (afas:38-106).  Returns the V-cycle count; the
// residual trace goes to `trace` (maxvcycles entries) when non-null.
int MultigridIterations(Ctx& c, double* last_residual, double* trace) {
  FillDown(c, false);
  for (int level = c.finestlevel; level >= Ctx::rootlevel; --level)
    for (Patch* p : c.on(level)) GetSourceFunction(c, *p);
  for (int level = c.finestlevel; level >= Ctx::rootlevel; --level)
    for (Patch* p : c.on(level)) UpdateSourceFunction(c, *p);
  FillDown(c, true);
  int itmg;
  double residual = 0.0;
  for (itmg = 1; itmg <= c.maxvcycles; ++itmg) {
    AFASVcycle(c, c.finestlevel);
    FillDown(c, false);
    for (int level = c.finestlevel; level >= Ctx::rootlevel; --level)
      for (Patch* p : c.on(level)) UpdateSourceFunction(c, *p);
    FillDown(c, true);
    residual = ErrorAFAS(c, c.finestlevel);
    if (trace) trace[itmg - 1] = residual;
    if (residual < c.qerrortol) break;
    // MultiGridUserBreak is .false. for this problem (problem.f90:814-821).
  }
  if (last_residual) *last_residual = residual;
  return itmg > c.maxvcycles ? c.maxvcycles : itmg;
}

void CopyQToQold(Patch& p) {
  if (p.tobedeleted) return;
  p.qold.d = p.q.d;
}

int resolve_minlevel(const orc_params* p) {
  if (p->minlevel != 1) return p->minlevel;
  int ml = 0, mxt[3] = {p->mx[0], p->mx[1], p->mx[2]};
  for (;;) {
    bool even = true;
    for (int n = 0; n < p->ndims; ++n) even = even && (mxt[n] % 2 == 0);
    if (!even) break;
    if (ml == 10) break;
    ++ml;
    for (int n = 0; n < p->ndims; ++n) mxt[n] /= 2;
  }
  return -ml;
}

// RootInit + CreateBelowSeedLevels + InitSeed (lib/bsamroutines.f90:205-494,
// lib/treeops.f90:193-289) for a single root grid with maxlevel = 0.
int BuildUniform(Ctx& c, const orc_params* p) {
  if (p->ndims < 2 || p->ndims > 3) return -1;
  if (p->errortype != 1) return -2;
  for (int n = 0; n < p->ndims; ++n) {
    if (p->mx[n] <= 0 || p->mx[n] % 2 != 0) return -3;
    if (p->xupper[n] <= p->xlower[n]) return -4;
  }
  // Physical (1, 10-99) or periodic (2, both faces of a dimension; the
  // reference stops on an unpaired periodic face, bsamroutines.f90:307-316).
  for (int f = 0; f < 2 * p->ndims; ++f) {
    int code = p->mthbc[f];
    if (code == 2) {
      if (p->mthbc[f ^ 1] != 2) return -5;
      c.periodic = true;
      continue;
    }
    if (!(code == 1 || (code >= 10 && code <= 99))) return -5;
  }
  c.ndims = p->ndims;
  c.dt = p->dt;
  c.qerrortol = p->qerrortol;
  c.alpha = p->alpha;
  c.eps = p->eps;
  c.eps2 = p->eps * p->eps;
  c.maxvcycles = p->maxvcycles;
  c.nsmoothingpasses = p->nsmoothingpasses;
  c.errortype = p->errortype;
  c.minlevel = resolve_minlevel(p);
  if (c.minlevel > 0 || c.minlevel < -10) return -6;
  c.finestlevel = 0;
  c.levels.assign(1 - c.minlevel, {});

  auto root = std::make_unique<Patch>();
  root->level = 0;
  for (int n = 0; n < c.ndims; ++n) {
    root->mx[n] = p->mx[n];
    root->mglobal[n][0] = 1;
    root->mglobal[n][1] = p->mx[n];
    root->mbounds[n][0] = 1;
    root->mbounds[n][1] = p->mx[n];
    root->xlower[n] = p->xlower[n];
    root->dx[n] = (p->xupper[n] - p->xlower[n]) / (double)p->mx[n];
  }
  for (int f = 0; f < 6; ++f) root->mthbc[f] = f < 2 * c.ndims ? p->mthbc[f] : 1;
  for (int n = 1; n < c.ndims; ++n)
    if (std::fabs(root->dx[0] - root->dx[n]) > 1.0e-10) return -7;
  AllocFields(c, *root);
  Patch* child = root.get();
  c.on(0).push_back(child);
  c.store.push_back(std::move(root));
  for (int level = -1; level >= c.minlevel; --level) {
    for (int n = 0; n < c.ndims; ++n)
      if (child->mx[n] % 2 != 0) return -8;
    auto seed = std::make_unique<Patch>();
    seed->level = level;
    for (int n = 0; n < c.ndims; ++n) {
      seed->mx[n] = child->mx[n] / 2;
      seed->dx[n] = child->dx[n] * 2.0;
      seed->mglobal[n][0] = 1;
      seed->mglobal[n][1] = child->mglobal[n][1] / 2;
      child->mbounds[n][0] = 1;
      child->mbounds[n][1] = seed->mx[n];
      seed->mbounds[n][0] = 1;
      seed->mbounds[n][1] = seed->mx[n];
      seed->xlower[n] = child->xlower[n];
    }
    for (int f = 0; f < 6; ++f) seed->mthbc[f] = child->mthbc[f];
    AllocFields(c, *seed);
    child->parent = seed.get();
    child = seed.get();
    c.on(level).push_back(child);
    c.store.push_back(std::move(seed));
  }
  return 0;
}

// A hierarchy given patch by patch (the caller's ApplyOnLevel order within
// each level): the nodeinfo fields the hot path reads, fields allocated.
int BuildFromPatches(Ctx& c, const orc_params* p, int npatch, const orc_patch* d) {
  if (p->ndims < 2 || p->ndims > 3 || p->errortype != 1 || npatch <= 0) return -1;
  // Periodic faces on a hierarchy given patch by patch are not restated
  // (TransferPeriodicBC between refined grids).
  for (int i = 0; i < npatch; ++i)
    for (int f = 0; f < 2 * p->ndims; ++f)
      if (d[i].mthbc[f] == 2) return -5;
  c.ndims = p->ndims;
  c.dt = p->dt;
  c.qerrortol = p->qerrortol;
  c.alpha = p->alpha;
  c.eps = p->eps;
  c.eps2 = p->eps * p->eps;
  c.maxvcycles = p->maxvcycles;
  c.nsmoothingpasses = p->nsmoothingpasses;
  c.errortype = p->errortype;
  int lo = d[0].level, hi = d[0].level;
  for (int i = 0; i < npatch; ++i) {
    lo = std::min(lo, d[i].level);
    hi = std::max(hi, d[i].level);
  }
  if (lo > 0 || hi < 0) return -2;
  c.minlevel = lo;
  c.finestlevel = hi;
  c.levels.assign(hi - lo + 1, {});
  std::vector<Patch*> made(npatch);
  for (int i = 0; i < npatch; ++i) {
    auto pt = std::make_unique<Patch>();
    pt->level = d[i].level;
    for (int n = 0; n < 3; ++n) {
      pt->mx[n] = n < c.ndims ? d[i].mx[n] : 1;
      for (int s = 0; s < 2; ++s) {
        pt->mbounds[n][s] = n < c.ndims ? d[i].mbounds[n][s] : 1;
        pt->mglobal[n][s] = n < c.ndims ? d[i].mglobal[n][s] : 1;
      }
      pt->dx[n] = d[i].dx;
      pt->xlower[n] = d[i].xlower[n];
    }
    for (int f = 0; f < 6; ++f) pt->mthbc[f] = f < 2 * c.ndims ? d[i].mthbc[f] : 1;
    AllocFields(c, *pt);
    made[i] = pt.get();
    c.on(pt->level).push_back(pt.get());
    c.store.push_back(std::move(pt));
  }
  for (int i = 0; i < npatch; ++i) {
    const int par = d[i].parent;
    if (par >= npatch || (par < 0 && d[i].level != lo)) return -3;
    if (par >= 0) {
      if (d[par].level != d[i].level - 1) return -3;
      made[i]->parent = made[par];
    }
  }
  return 0;
}

// Wrap a flat Fortran-ordered array into an FArr with the given bounds.
FArr wrap(int ndims, const int* lo, const int* hi, int nv, const double* src) {
  FArr a;
  a.alloc(lo[0], hi[0], lo[1], hi[1], ndims == 3 ? lo[2] : 1, ndims == 3 ? hi[2] : 1, 1, nv);
  if (src) std::memcpy(a.d.data(), src, a.d.size() * sizeof(double));
  return a;
}

Ctx leaf_ctx(int ndims, double dt, double alpha, double eps) {
  Ctx c;
  c.ndims = ndims;
  c.dt = dt;
  c.alpha = alpha;
  c.eps = eps;
  c.eps2 = eps * eps;
  return c;
}

}  // namespace

// ---------------------------------------------------------------------------
extern "C" {

int orc_minlevel(const orc_params* p) { return resolve_minlevel(p); }

int orc_run_uniform(const orc_params* p, const double* q0, int nsteps, double* q_steps,
                    int* nvcycles, double* resid_final, double* resid_trace, double* mass) {
  Ctx c;
  int err = BuildUniform(c, p);
  if (err) return err;
  Patch& root = *c.on(0)[0];
  std::memcpy(root.q.d.data(), q0, root.q.d.size() * sizeof(double));
  // BSAMSolver: SetGhost(rootlevel,0); CopyQToQold (bsamroutines.f90:144-147).
  if (SetGhost(c, 0, 0)) return -9;
  CopyQToQold(root);
  bool firstamr = true;
  double h = root.dx[0];
  for (int step = 0; step < nsteps; ++step) {
    c.finestlevel = 0;
    SetGhost(c, 0, 0);  // AMR(rootlevel) with maxlevel = 0
    if (firstamr) {
      FillDown(c, false);
      firstamr = false;
    }
    for (int level = c.minlevel; level <= c.finestlevel; ++level)
      for (Patch* pp : c.on(level)) CopyQToQold(*pp);
    double* tr = resid_trace ? resid_trace + (long)step * c.maxvcycles : nullptr;
    if (tr)
      for (int i = 0; i < c.maxvcycles; ++i) tr[i] = -1.0;
    double last = 0.0;
    int nv = MultigridIterations(c, &last, tr);
    if (nvcycles) nvcycles[step] = nv;
    if (resid_final) resid_final[step] = last;
    if (q_steps)
      std::memcpy(q_steps + (long)step * root.q.d.size(), root.q.d.data(),
                  root.q.d.size() * sizeof(double));
    if (mass) {
      // AfterStep2D/3D, level 0 (problem.f90:121-122, 416-418).
      double s = 0.0;
      int n3 = c.ndims == 3 ? root.mx[2] : 1;
      for (int k = 1; k <= n3; ++k)
        for (int j = 1; j <= root.mx[1]; ++j)
          for (int i = 1; i <= root.mx[0]; ++i) s = s + root.q(i, j, k, 1);
      double hd = c.ndims == 2 ? h * h : h * h * h;
      mass[step] = hd * s;
    }
  }
  return 0;
}

// ---- a hierarchy held between calls (regridding runs) ----------------------
struct orc_hier {
  Ctx c;
  std::vector<Patch*> byindex;  // patch table order
};

orc_hier* orc_hier_create(const orc_params* p, int npatch, const orc_patch* patches) {
  auto* H = new orc_hier();
  if (BuildFromPatches(H->c, p, npatch, patches)) {
    delete H;
    return nullptr;
  }
  for (auto& up : H->c.store) H->byindex.push_back(up.get());
  return H;
}
void orc_hier_destroy(orc_hier* H) { delete H; }
int orc_hier_q(orc_hier* H, int patch, double* q, int put) {
  if (!H || patch < 0 || patch >= (int)H->byindex.size()) return -1;
  Patch& P = *H->byindex[patch];
  if (put) std::memcpy(P.q.d.data(), q, P.q.d.size() * sizeof(double));
  else std::memcpy(q, P.q.d.data(), P.q.d.size() * sizeof(double));
  return 0;
}
int orc_hier_set_ghost(orc_hier* H, int level) {
  if (!H || level < H->c.minlevel || level > H->c.finestlevel) return -1;
  return SetGhost(H->c, level, 0);
}
// RestrictSolution of a refined level into its parents (FillDownLevel's
// expression, the same values) and the parent level's SetGhost.
int orc_hier_restrict_level(orc_hier* H, int level) {
  if (!H || level < 1 || level > H->c.finestlevel) return -1;
  for (Patch* p : H->c.on(level)) FillDownLevel(H->c, *p, false);
  return SetGhost(H->c, level - 1, 0);
}
int orc_hier_fill_down(orc_hier* H) {
  if (!H) return -1;
  FillDown(H->c, false);
  return 0;
}
int orc_hier_copy_q_to_qold(orc_hier* H) {
  if (!H) return -1;
  for (int level = H->c.minlevel; level <= H->c.finestlevel; ++level)
    for (Patch* pp : H->c.on(level)) CopyQToQold(*pp);
  return 0;
}
int orc_hier_multigrid(orc_hier* H, int* nvcycles, double* residual) {
  if (!H) return -1;
  double last = 0.0;
  const int nv = MultigridIterations(H->c, &last, nullptr);
  if (nvcycles) *nvcycles = nv;
  if (residual) *residual = last;
  return 0;
}

// AfterStepStatistics (lib/bsamroutines.f90:893-937) with AfterStep2D/3D
// (problem.f90:102-134, 398-424): levels finestlevel down to rootlevel,
// ApplyOnLevel order; on a refined patch, qc is the parent's q over
// mbounds - 1 .. mbounds + 1.
int orc_hier_after_step(orc_hier* H, double* integral) {
  if (!H || !integral) return -1;
  Ctx& c = H->c;
  const int nd = c.ndims;
  double r1 = 0.0, r2 = 0.0;
  // Column-major sum of c over [lo, hi] of patch P (Fortran sum).
  auto csum = [&](Patch& P, const int* lo, const int* hi) {
    double s = 0.0;
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int j = lo[1]; j <= hi[1]; ++j)
        for (int i = lo[0]; i <= hi[0]; ++i) s = s + P.q(i, j, k, 1);
    return s;
  };
  // Energy2D of c over [lo - 1, hi + 1] of P (a copy, then the leaf routine).
  auto energy = [&](Patch& P, const int* lo, const int* hi, double h) {
    const int n1 = hi[0] - lo[0] + 1, n2 = hi[1] - lo[1] + 1;
    std::vector<double> a((size_t)(n1 + 2) * (n2 + 2));
    for (int j = 0; j <= n2 + 1; ++j)
      for (int i = 0; i <= n1 + 1; ++i)
        a[(size_t)i + (size_t)(n1 + 2) * j] = P.q(lo[0] - 1 + i, lo[1] - 1 + j, 1, 1);
    const int mx[2] = {n1, n2};
    return orc_energy2d(mx, h, c.alpha, c.eps, a.data());
  };
  for (int level = c.finestlevel; level >= 0; --level) {
    for (Patch* pp : c.on(level)) {
      Patch& P = *pp;
      const double h = P.dx[0], ch = h * 2.0;
      int lo[3] = {1, 1, 1}, hi[3] = {P.mx[0], P.mx[1], nd == 3 ? P.mx[2] : 1};
      int clo[3] = {1, 1, 1}, chi[3] = {1, 1, 1};
      for (int n = 0; n < nd; ++n) {
        clo[n] = P.mbounds[n][0];
        chi[n] = P.mbounds[n][1];
      }
      if (nd == 2) {
        const double h2 = h * h, ch2 = ch * ch;
        if (level == 0) {
          r1 = r1 + h2 * csum(P, lo, hi);
          r2 = r2 + energy(P, lo, hi, h);
        } else {
          r1 = r1 + h2 * csum(P, lo, hi) - ch2 * csum(*P.parent, clo, chi);
          r2 = r2 + energy(P, lo, hi, h) - energy(*P.parent, clo, chi, ch);
        }
      } else {
        const double h3 = h * h * h, ch3 = ch * ch * ch;
        if (level == 0) r1 = r1 + h3 * csum(P, lo, hi);
        else r1 = r1 + h3 * csum(P, lo, hi) - ch3 * csum(*P.parent, clo, chi);
      }
    }
  }
  integral[0] = r1;
  integral[1] = r2;
  return 0;
}

int orc_run_hier(const orc_params* p, int npatch, const orc_patch* patches, const double* q0,
                 int nsteps, double* q_out, int* nvcycles, double* resid_final) {
  Ctx c;
  int err = BuildFromPatches(c, p, npatch, patches);
  if (err) return err;
  // q of the patches on levels >= root, in input order, each with its ring.
  auto each_state = [&](auto fn) {
    size_t off = 0;
    for (auto& up : c.store) {
      Patch& pt = *up;
      if (pt.level < Ctx::rootlevel) continue;
      fn(pt, off);
      off += pt.q.d.size();
    }
  };
  each_state([&](Patch& pt, size_t off) {
    std::memcpy(pt.q.d.data(), q0 + off, pt.q.d.size() * sizeof(double));
  });
  // Start (BSAMSolver, bsamroutines.f90:144-147) and every step: the ghosts
  // of every level from the root up, as AMR(rootlevel) leaves them on an
  // unchanged hierarchy; then FillDown once, CopyQToQold and
  // MultigridIterations (TakeTimeSteps, bsamroutines.f90:648-723).
  auto ghosts = [&]() {
    for (int level = Ctx::rootlevel; level <= c.finestlevel; ++level)
      if (SetGhost(c, level, 0)) return -9;
    return 0;
  };
  if (ghosts()) return -9;
  for (int level = c.minlevel; level <= c.finestlevel; ++level)
    for (Patch* pp : c.on(level)) CopyQToQold(*pp);
  bool firstamr = true;
  for (int step = 0; step < nsteps; ++step) {
    if (ghosts()) return -9;
    if (firstamr) {
      FillDown(c, false);
      firstamr = false;
    }
    for (int level = c.minlevel; level <= c.finestlevel; ++level)
      for (Patch* pp : c.on(level)) CopyQToQold(*pp);
    double last = 0.0;
    const int nv = MultigridIterations(c, &last, nullptr);
    if (nvcycles) nvcycles[step] = nv;
    if (resid_final) resid_final[step] = last;
  }
  if (q_out)
    each_state([&](Patch& pt, size_t off) {
      std::memcpy(q_out + off, pt.q.d.data(), pt.q.d.size() * sizeof(double));
    });
  return 0;
}

void orc_interpolate3d(const int* mx, int nv, const int* mbounds, const int* mthbc, int ipass,
                       double* qf, const int* pmx, const double* qc) {
  const int lo[3] = {0, 0, 0};
  const int hi[3] = {mx[0] + 1, mx[1] + 1, mx[2] + 1};
  const int phi[3] = {pmx[0] + 1, pmx[1] + 1, pmx[2] + 1};
  FArr f = wrap(3, lo, hi, nv, qf);
  FArr c = wrap(3, lo, phi, nv, qc);
  const int mb[3][2] = {{mbounds[0], mbounds[1]}, {mbounds[2], mbounds[3]},
                        {mbounds[4], mbounds[5]}};
  Interpolate3D(f, c, mx, nv, mb, mthbc, ipass);
  std::memcpy(qf, f.d.data(), f.d.size() * sizeof(double));
}

void orc_interpolate2d(const int* mx, int nv, const int* mbounds, const int* mthbc, int ipass,
                       double* qf, const int* pmx, const double* qc) {
  int lo[3] = {0, 0, 1}, hi[3] = {mx[0] + 1, mx[1] + 1, 1};
  int plo[3] = {0, 0, 1}, phi[3] = {pmx[0] + 1, pmx[1] + 1, 1};
  FArr F = wrap(2, lo, hi, nv, qf), C = wrap(2, plo, phi, nv, qc);
  int mb[3][2] = {{mbounds[0], mbounds[1]}, {mbounds[2], mbounds[3]}, {1, 1}};
  Interpolate2D(F, C, mx, nv, mb, mthbc, ipass);
  std::memcpy(qf, F.d.data(), F.d.size() * sizeof(double));
}

void orc_relax_grid(int ndims, const int* mx, double h, double dt, double alpha, double eps,
                    int ipass, double* q, const double* f) {
  Ctx c = leaf_ctx(ndims, dt, alpha, eps);
  int lo[3] = {0, 0, 0}, hi[3] = {mx[0] + 1, mx[1] + 1, ndims == 3 ? mx[2] + 1 : 1};
  int flo[3] = {1, 1, 1}, fhi[3] = {mx[0], mx[1], ndims == 3 ? mx[2] : 1};
  FArr Q = wrap(ndims, lo, hi, 2, q), F = wrap(ndims, flo, fhi, 2, f);
  if (ndims == 2) RelaxGrid2D(c, Q, F, mx, h, ipass);
  else RelaxGrid3D(c, Q, F, mx, h, ipass);
  std::memcpy(q, Q.d.data(), Q.d.size() * sizeof(double));
}

void orc_operator(int ndims, const int* mx, double h, double dt, double alpha, double eps,
                  const double* q, double* res) {
  Ctx c = leaf_ctx(ndims, dt, alpha, eps);
  int lo[3] = {0, 0, 0}, hi[3] = {mx[0] + 1, mx[1] + 1, ndims == 3 ? mx[2] + 1 : 1};
  FArr Q = wrap(ndims, lo, hi, 2, q), R;
  Operator(c, Q, mx, h, R);
  std::memcpy(res, R.d.data(), R.d.size() * sizeof(double));
}

void orc_restriction(int ndims, const int* mx, int nv, const double* a, double* out) {
  Ctx c = leaf_ctx(ndims, 0, 1, 0);
  int lo[3] = {1, 1, 1}, hi[3] = {mx[0], mx[1], ndims == 3 ? mx[2] : 1};
  FArr A = wrap(ndims, lo, hi, nv, a), O;
  Restriction(c, A, mx, nv, O);
  std::memcpy(out, O.d.data(), O.d.size() * sizeof(double));
}

void orc_prolongation_p1(int ndims, const int* cmx, int nv, const double* a, double* out) {
  Ctx c = leaf_ctx(ndims, 0, 1, 0);
  int lo[3] = {0, 0, 0}, hi[3] = {cmx[0] + 1, cmx[1] + 1, ndims == 3 ? cmx[2] + 1 : 1};
  FArr A = wrap(ndims, lo, hi, nv, a), O;
  ProlongationP1(c, A, cmx, nv, O);
  std::memcpy(out, O.d.data(), O.d.size() * sizeof(double));
}

int orc_setbc(int ndims, const int* mx, int nv, const int* mthbc, double* q) {
  int lo[3] = {0, 0, 0}, hi[3] = {mx[0] + 1, mx[1] + 1, ndims == 3 ? mx[2] + 1 : 1};
  FArr Q = wrap(ndims, lo, hi, nv, q);
  int err = ndims == 2 ? SetBC2D(Q, mx, nv, mthbc) : SetBC3D(Q, mx, nv, mthbc);
  std::memcpy(q, Q.d.data(), Q.d.size() * sizeof(double));
  return err;
}

void orc_source(int ndims, const int* mx, double alpha, const double* qold, double* f) {
  Ctx c = leaf_ctx(ndims, 0, alpha, 0);
  Patch p;
  p.mx[0] = mx[0];
  p.mx[1] = mx[1];
  p.mx[2] = ndims == 3 ? mx[2] : 1;
  AllocFields(c, p);
  std::memcpy(p.qold.d.data(), qold, p.qold.d.size() * sizeof(double));
  GetSourceFunction(c, p);
  std::memcpy(f, p.ftmp.d.data(), p.ftmp.d.size() * sizeof(double));
}

// SetErrFlagsUser2D / 3D (problem.f90:135-163, 425-452): a cell is flagged
// where the undivided central gradient of c exceeds tol.  q: c with its ring,
// (0:mx+1)^d; flags (1:mx)^d.
void orc_errflags(int ndims, const int* mx, double tol, const double* q, int* flags) {
  const int n0 = mx[0], n1 = mx[1], n2 = ndims == 3 ? mx[2] : 1;
  const long s1 = n0 + 2, s2 = (long)(n0 + 2) * (n1 + 2);
  auto C = [&](int i, int j, int k) { return q[i + s1 * j + (ndims == 3 ? s2 * k : 0)]; };
  long o = 0;
  for (int k = 1; k <= n2; ++k)
    for (int j = 1; j <= n1; ++j)
      for (int i = 1; i <= n0; ++i) {
        const double dx = C(i + 1, j, k) - C(i - 1, j, k), dy = C(i, j + 1, k) - C(i, j - 1, k);
        double s = dx * dx + dy * dy;
        if (ndims == 3) {
          const double dz = C(i, j, k + 1) - C(i, j, k - 1);
          s = s + dz * dz;
        }
        flags[o++] = std::fabs(std::sqrt(s)) > tol ? 1 : 0;
      }
}

// Bi/TriLinProlongationP1MC (gridutilities.f90:219-279, 588-686): linear
// prolongation one direction after the other, then each coarse cell's mass
// correction cor = a - (average of its children) added to every child.
// a: (0:cmx+1)^d x nv, out: (0:2cmx+1)^d x nv.
void orc_prolong_mc(int ndims, const int* cmx, int nv, const double* ain, double* out) {
  const int lo[3] = {0, 0, 0};
  const int ahi[3] = {cmx[0] + 1, cmx[1] + 1, ndims == 3 ? cmx[2] + 1 : 0};
  FArr A = wrap(ndims, lo, ahi, nv, ain);
  const int m0 = 2 * cmx[0], m1 = 2 * cmx[1], m2 = ndims == 3 ? 2 * cmx[2] : 0;
  const int c0 = cmx[0], c1 = cmx[1], c2 = ndims == 3 ? cmx[2] : 0;
  const int kk = ndims == 3 ? 0 : 1;  // the third index of 2D arrays
  FArr B, Cc, P;
  if (ndims == 2) {
    B.alloc(0, m0 + 1, 0, c1 + 1, 1, 1, 1, nv);
    P.alloc(0, m0 + 1, 0, m1 + 1, 1, 1, 1, nv);
  } else {
    B.alloc(0, m0 + 1, 0, c1 + 1, 0, c2 + 1, 1, nv);
    Cc.alloc(0, m0 + 1, 0, m1 + 1, 0, c2 + 1, 1, nv);
    P.alloc(0, m0 + 1, 0, m1 + 1, 0, m2 + 1, 1, nv);
  }
  const int k3 = ndims == 3 ? c2 + 1 : kk;
  for (int v = 1; v <= nv; ++v)
    for (int k = ndims == 3 ? 0 : 1; k <= k3; ++k)
      for (int j = 0; j <= c1 + 1; ++j)
        for (int i = 0; i <= c0; ++i) {
          B(2 * i, j, k, v) = 3.0 * A(i, j, k, v) + A(i + 1, j, k, v);
          B(2 * i + 1, j, k, v) = A(i, j, k, v) + 3.0 * A(i + 1, j, k, v);
        }
  if (ndims == 2) {
    for (int v = 1; v <= nv; ++v)
      for (int j = 0; j <= c1; ++j)
        for (int i = 0; i <= m0 + 1; ++i) {
          P(i, 2 * j, 1, v) = (3.0 * B(i, j, 1, v) + B(i, j + 1, 1, v)) / 16.0;
          P(i, 2 * j + 1, 1, v) = (B(i, j, 1, v) + 3.0 * B(i, j + 1, 1, v)) / 16.0;
        }
    for (int v = 1; v <= nv; ++v)
      for (int l = 1; l <= c1; ++l)
        for (int k = 1; k <= c0; ++k) {
          const double cor = A(k, l, 1, v) - 0.25 * (P(2 * k, 2 * l, 1, v) + P(2 * k - 1, 2 * l, 1, v) +
                                                     P(2 * k, 2 * l - 1, 1, v) +
                                                     P(2 * k - 1, 2 * l - 1, 1, v));
          P(2 * k, 2 * l, 1, v) = P(2 * k, 2 * l, 1, v) + cor;
          P(2 * k - 1, 2 * l, 1, v) = P(2 * k - 1, 2 * l, 1, v) + cor;
          P(2 * k, 2 * l - 1, 1, v) = P(2 * k, 2 * l - 1, 1, v) + cor;
          P(2 * k - 1, 2 * l - 1, 1, v) = P(2 * k - 1, 2 * l - 1, 1, v) + cor;
        }
  } else {
    for (int v = 1; v <= nv; ++v)
      for (int k = 0; k <= c2 + 1; ++k)
        for (int j = 0; j <= c1; ++j)
          for (int i = 0; i <= m0 + 1; ++i) {
            Cc(i, 2 * j, k, v) = 3.0 * B(i, j, k, v) + B(i, j + 1, k, v);
            Cc(i, 2 * j + 1, k, v) = B(i, j, k, v) + 3.0 * B(i, j + 1, k, v);
          }
    for (int v = 1; v <= nv; ++v)
      for (int k = 0; k <= c2; ++k)
        for (int j = 0; j <= m1 + 1; ++j)
          for (int i = 0; i <= m0 + 1; ++i) {
            P(i, j, 2 * k, v) = (3.0 * Cc(i, j, k, v) + Cc(i, j, k + 1, v)) / 64.0;
            P(i, j, 2 * k + 1, v) = (Cc(i, j, k, v) + 3.0 * Cc(i, j, k + 1, v)) / 64.0;
          }
    for (int v = 1; v <= nv; ++v)
      for (int n = 1; n <= c2; ++n)
        for (int l = 1; l <= c1; ++l)
          for (int k = 1; k <= c0; ++k) {
            const int a = 2 * k, b = 2 * l, c = 2 * n;
            const double cor =
                A(k, l, n, v) - 0.125 * (P(a, b, c, v) + P(a - 1, b, c, v) + P(a, b - 1, c, v) +
                                         P(a - 1, b - 1, c, v) + P(a, b, c - 1, v) +
                                         P(a - 1, b, c - 1, v) + P(a, b - 1, c - 1, v) +
                                         P(a - 1, b - 1, c - 1, v));
            for (int dz = 0; dz < 2; ++dz)
              for (int dy = 0; dy < 2; ++dy)
                for (int dx = 0; dx < 2; ++dx)
                  P(a - dx, b - dy, c - dz, v) = P(a - dx, b - dy, c - dz, v) + cor;
          }
  }
  std::memcpy(out, P.d.data(), P.d.size() * sizeof(double));
}

// NewSubGrids (lib/bsamroutines.f90:1352-1528) with GetSignatures
// (1530-1554) and GridFlagRatio (1556-1579): Berger-Rigoutsos clustering of
// the flags of a patch (1:mx)^d into boxes of at least mgp cells per side
// whose flagged fraction reaches desfill where splits allow.  Boxes go to
// `boxes` (per box lo/hi per dimension, 3 x 2 ints, dimensions beyond d = 1)
// in the order the reference makes the new grids; returns their number, or
// -1 if more than maxboxes.
int orc_new_subgrids(int ndims, const int* mx, const int* flags, double desfill, int mgp,
                     int* boxes, int maxboxes) {
  constexpr int maxsubgrids = 1024, maxsplitpasses = 15;
  const int nd = ndims;
  const int m[3] = {mx[0], mx[1], nd == 3 ? mx[2] : 1};
  auto F = [&](int i, int j, int k) {
    return flags[(i - 1) + (long)m[0] * ((j - 1) + (long)m[1] * (k - 1))];
  };
  auto box_sum = [&](const int lo[3], const int hi[3]) {
    long s = 0;
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int j = lo[1]; j <= hi[1]; ++j)
        for (int i = lo[0]; i <= hi[0]; ++i) s += F(i, j, k);
    return s;
  };
  // GridFlagRatio: real(flagged) / real(product of extents).
  auto ratio = [&](int (*mb)[2]) {
    double total = 1.0;
    long prod = 1;
    for (int n = 0; n < nd; ++n) prod *= (mb[n][1] - mb[n][0] + 1);
    total = (double)prod;
    for (int n = nd; n < 3; ++n) mb[n][0] = mb[n][1] = 1;
    const int lo[3] = {mb[0][0], mb[1][0], mb[2][0]}, hi[3] = {mb[0][1], mb[1][1], mb[2][1]};
    return (double)box_sum(lo, hi) / total;
  };
  int maxm = 0;
  for (int n = 0; n < nd; ++n) maxm = std::max(maxm, m[n]);
  std::vector<long> sig((size_t)(maxm + 2) * 3, 0), dd((size_t)(maxm + 2) * 3, 0);
  auto S = [&](int i, int n) -> long& { return sig[(size_t)i + (size_t)(maxm + 2) * n]; };
  auto DD = [&](int i, int n) -> long& { return dd[(size_t)i + (size_t)(maxm + 2) * n]; };
  // GetSignatures over box g.
  auto signatures = [&](int (*mb)[2]) {
    for (int n = 0; n < nd; ++n) {
      int lo[3] = {1, 1, 1}, hi[3] = {1, 1, 1};
      for (int d = 0; d < nd; ++d) {
        lo[d] = mb[d][0];
        hi[d] = mb[d][1];
      }
      for (int i = mb[n][0]; i <= mb[n][1]; ++i) {
        lo[n] = hi[n] = i;
        S(i, n) = box_sum(lo, hi);
      }
    }
  };
  int whole[3][2] = {{1, m[0]}, {1, m[1]}, {1, m[2]}};
  if (ratio(whole) < 1.0e-10) return 0;
  std::vector<std::array<std::array<int, 2>, 3>> sub(maxsubgrids + 1);
  std::vector<char> cansplit(maxsubgrids + 1, 1);
  int ngrid = 1;
  for (int n = 0; n < 3; ++n) sub[1][n] = {whole[n][0], whole[n][1]};
  int igrid = 1;
  while (ngrid < maxsubgrids && igrid <= ngrid) {
    int npass = 0;
    while (cansplit[igrid] && npass < maxsplitpasses) {
      ++npass;
      int mb[3][2];
      auto load = [&]() {
        for (int n = 0; n < 3; ++n) {
          mb[n][0] = sub[igrid][n][0];
          mb[n][1] = sub[igrid][n][1];
        }
      };
      auto store = [&]() {
        for (int n = 0; n < 3; ++n) sub[igrid][n] = {mb[n][0], mb[n][1]};
      };
      load();
      signatures(mb);
      // Trim empty rows and columns at the box's ends.
      for (int n = 0; n < nd; ++n) {
        int i1 = mb[n][0], i2 = mb[n][1];
        while (S(i1, n) == 0 && i1 < mb[n][1] && i2 - i1 + 1 > mgp) ++i1;
        while (S(i2, n) == 0 && i2 > mb[n][0] && i2 - i1 + 1 > mgp) --i2;
        mb[n][0] = i1;
        mb[n][1] = i2;
      }
      const double fill = ratio(mb);
      store();
      if (fill < desfill) {
        signatures(mb);
        int isplit[3] = {0, 0, 0};
        bool havesplit = false;
        // A hole: a zero signature at least mgp from both ends.
        for (int n = 0; n < nd && !havesplit; ++n) {
          const int i1 = mb[n][0], i2 = mb[n][1];
          for (int i = i1 + mgp; i <= i2 - mgp; ++i)
            if (S(i, n) == 0 && std::min(i - i1 + 1, i2 - i) >= mgp) {
              isplit[n] = i;
              havesplit = true;
              break;
            }
        }
        if (!havesplit) {
          // The strongest inflection of the signature (ties: the most central).
          for (int n = 0; n < nd; ++n) {
            const int i1 = mb[n][0], i2 = mb[n][1];
            for (int i = i1 + 1; i <= i2 - 1; ++i) DD(i, n) = S(i - 1, n) - 2 * S(i, n) + S(i + 1, n);
          }
          long inflect = 0;
          int dist0 = 0;
          for (int n = 0; n < nd; ++n) {
            const int i1 = mb[n][0], i2 = mb[n][1];
            for (int i = i1 + std::max(2, mgp); i <= i2 - std::max(1, mgp - 1); ++i) {
              const long del = std::labs(DD(i, n) - DD(i - 1, n));
              if (del > inflect) {
                inflect = del;
                isplit[0] = isplit[1] = isplit[2] = 0;
                isplit[n] = i - 1;
                havesplit = true;
                dist0 = std::min(i - i1, i2 - i + 1);
              } else if (del == inflect && inflect > 0) {
                const int dist1 = std::min(i - i1, i2 - i + 1);
                if (dist1 > dist0) {
                  isplit[0] = isplit[1] = isplit[2] = 0;
                  isplit[n] = i - 1;
                  havesplit = true;
                  dist0 = dist1;
                }
              }
            }
          }
        }
        if (havesplit) {
          for (int n = 0; n < nd; ++n)
            if (isplit[n] > 0 &&
                std::min(sub[igrid][n][1] - isplit[n], isplit[n] - sub[igrid][n][0] + 1) >= mgp) {
              ++ngrid;
              cansplit[ngrid] = 1;
              sub[ngrid] = sub[igrid];
              sub[ngrid][n][0] = isplit[n] + 1;
              sub[igrid][n][1] = isplit[n];
              break;
            }
        } else {
          cansplit[igrid] = 0;
        }
      } else {
        cansplit[igrid] = 0;
      }
    }
    ++igrid;
  }
  if (ngrid > maxboxes) return -1;
  for (int g = 1; g <= ngrid; ++g)
    for (int n = 0; n < 3; ++n) {
      boxes[(g - 1) * 6 + 2 * n] = n < nd ? sub[g][n][0] : 1;
      boxes[(g - 1) * 6 + 2 * n + 1] = n < nd ? sub[g][n][1] : 1;
    }
  return ngrid;
}

double orc_energy2d(const int* mx, double h, double alpha, double eps, const double* cin) {
  // Energy2D (problem.f90:330-361).
  Ctx c = leaf_ctx(2, 0, alpha, eps);
  int lo[3] = {0, 0, 1}, hi[3] = {mx[0] + 1, mx[1] + 1, 1};
  FArr C = wrap(2, lo, hi, 1, cin);
  int n1 = mx[0], n2 = mx[1];
  double h2 = h * h;
  FArr f1, f2;
  f1.alloc(0, n1, 1, n2, 1, 1, 1, 1);
  f2.alloc(1, n1, 0, n2, 1, 1, 1, 1);
  for (int j = 1; j <= n2; ++j)
    for (int i = 0; i <= n1; ++i) {
      double d = C(i + 1, j, 1, 1) - C(i, j, 1, 1);
      f1(i, j, 1, 1) = d * d;
    }
  for (int j = 0; j <= n2; ++j)
    for (int i = 1; i <= n1; ++i) {
      double d = C(i, j + 1, 1, 1) - C(i, j, 1, 1);
      f2(i, j, 1, 1) = d * d;
    }
  double tmp = c.eps2 / h2 / 4.0;
  double sF = 0.0, sG = 0.0;
  for (int j = 1; j <= n2; ++j)
    for (int i = 1; i <= n1; ++i) sF = sF + Ff(c, C(i, j, 1, 1));
  for (int j = 1; j <= n2; ++j)
    for (int i = 1; i <= n1; ++i)
      sG = sG + (f1(i, j, 1, 1) + f1(i - 1, j, 1, 1) + f2(i, j, 1, 1) + f2(i, j - 1, 1, 1));
  return h2 * (sF + tmp * sG);
}

}  // extern "C"
