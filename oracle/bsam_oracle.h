/*
 * bsam_oracle.h -- C API of the CPU oracle (TEST INFRASTRUCTURE ONLY).
 *
 * The oracle is a plain C++ restatement of the BSAM Fortran FAS multigrid
 * hot path for the simple_cahn-hilliard problem module.  It exists so that
 * tests, __graft_entry__.smoke() and bench.py's cpu_baseline leg can check
 * the CUDA path; the product never links, loads or calls it.
 *
 * Parity pinning: the reference is Fortran 90, no Fortran compiler exists in
 * this image, and the reference ships no tests or golden outputs.  The oracle
 * is PINNED bit for bit against fixtures produced by executing the
 * reference's own Fortran source with a Fortran-subset interpreter
 * (tests/golden/make_golden.py, tests/test_golden_reference.py): the leaf
 * routines (relaxation, operator, source, restriction, P1 prolongation,
 * SetBC/UserBC, Interpolate2D) and their composition, MultigridIterations
 * with the V-cycle, SetGhost, FillDown and ErrorAFAS (afasroutines.f90,
 * boundary.f90), on uniform 2D / 3D hierarchies and a 2D hierarchy with two
 * refined levels; and the regridding leaves: SetErrFlagsUser2D/3D, the
 * mass-corrected prolongation of InitFields, NewSubGrids (Berger-Rigoutsos)
 * and, in oracle/pyoracle.py, BufferAndList + InflateEdgeTags.  Restated
 * rather than interpreted on both sides: TreeOps' level traversal order,
 * TakeTimeSteps' step sequence, and the regridding composition (AMR,
 * EstimateLevelErrors, GridAdapt with MakeNewGrid's geometry and
 * TransferValues; bsamroutines.f90:632-723, 939-1002, 1299-1350, 1582-1867),
 * which the engine and the oracle run through one driver.  The interpreter
 * evaluates as the Fortran text reads, with no fused
 * multiply-add; a reference build that contracts a*b+c into FMA would differ
 * from it in the last bits.
 *
 * Array layout (every array argument): Fortran column-major, i fastest, with
 * the reference's bounds -- q(0:mx1+1, 0:mx2+1[, 0:mx3+1], 1:2) with the ghost
 * ring, f(1:mx1, 1:mx2[, 1:mx3], 1:2) without it (lib/bsamstorage.f90:74-102).
 */
#ifndef BSAM_ORACLE_H
#define BSAM_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int32_t ndims;            /* 2 or 3 */
  int32_t mx[3];            /* root-level interior cells per dimension */
  int32_t mthbc[6];         /* boundary code per face (1 Neumann, 10-99 user) */
  int32_t minlevel;         /* <= 0, or 1 for the automatic choice */
  int32_t nsmoothingpasses; /* nu of V(nu,nu) */
  int32_t maxvcycles;
  int32_t errortype;        /* only 1 is supported */
  int32_t pad_;
  double xlower[3], xupper[3];
  double dt, qerrortol, alpha, eps;
} orc_params;

/* Uniform-grid time stepping (maxlevel = 0): restates BSAMSolver ->
 * TakeTimeSteps -> MultigridIterations (lib/bsamroutines.f90:51-176,
 * 582-789; lib/afasroutines.f90:38-106) for nsteps steps with eqfn = 1.
 * q0: root q with ghost ring (the ring is recomputed by SetGhost).
 * Outputs (any may be NULL):
 *   q_steps       nsteps x size(q) -- root q (with ring) after each step
 *   nvcycles      nsteps           -- V-cycles performed per step
 *   resid_final   nsteps           -- last residual of each step
 *   resid_trace   nsteps x maxvcycles (unused entries set to -1)
 *   mass          nsteps           -- h^d * sum(phi) after each step
 * Returns 0, or a negative code for invalid parameters.               */
int orc_run_uniform(const orc_params* p, const double* q0, int nsteps,
                    double* q_steps, int* nvcycles, double* resid_final,
                    double* resid_trace, double* mass);

/* One patch of a given hierarchy (the nodeinfo fields the hot path reads,
 * lib/nodeinfodef.f90:124-219); parent is an index into the same array. */
typedef struct {
  int32_t level, parent, mx[3], mbounds[3][2], mglobal[3][2], mthbc[6];
  double dx, xlower[3];
} orc_patch;

/* Time stepping on a fixed hierarchy, AMR levels included (2D): every step
 * SetGhost(level, 0) from the root up (what AMR(rootlevel) leaves on an
 * unchanged hierarchy), FillDown(solution) on the first step, CopyQToQold,
 * MultigridIterations.  p supplies the run parameters (its mx, mthbc,
 * minlevel and bounds are not used).  q0 / q_out: q with ghost ring of every
 * patch on a level >= 0, concatenated in array order.  Returns 0 or a
 * negative code. */
int orc_run_hier(const orc_params* p, int npatch, const orc_patch* patches,
                 const double* q0, int nsteps, double* q_out, int* nvcycles,
                 double* resid_final);

/* A hierarchy held between calls, for regridding runs driven from outside:
 * the patch table as orc_run_hier takes it; q of any patch (with ring) put
 * or got (put != 0: q -> patch); SetGhost of one level; RestrictSolution of
 * a refined level into its parents followed by the parent level's SetGhost;
 * FillDown(solution); CopyQToQold on every level; MultigridIterations. */
typedef struct orc_hier orc_hier;
orc_hier* orc_hier_create(const orc_params* p, int npatch, const orc_patch* patches);
void orc_hier_destroy(orc_hier* h);
int orc_hier_q(orc_hier* h, int patch, double* q, int put);
int orc_hier_set_ghost(orc_hier* h, int level);
int orc_hier_restrict_level(orc_hier* h, int level);
int orc_hier_fill_down(orc_hier* h);
int orc_hier_copy_q_to_qold(orc_hier* h);
int orc_hier_multigrid(orc_hier* h, int* nvcycles, double* residual);
/* AfterStepStatistics over the held hierarchy: integral[0] the composite
 * mass, integral[1] the composite Energy2D (0 in 3D). */
int orc_hier_after_step(orc_hier* h, double* integral);

/* Interpolate2D (boundary.f90:135-323) on a fine patch qf (0:mx+1)^2 x nv
 * from its parent qc (0:pmx+1)^2 x nv; mbounds = {mb11, mb12, mb21, mb22}. */
void orc_interpolate2d(const int* mx, int nv, const int* mbounds, const int* mthbc,
                       int ipass, double* qf, const int* pmx, const double* qc);

/* Interpolate3D (boundary.f90:1299-1799) on a fine patch qf (0:mx+1)^3 x nv
 * from its parent qc (0:pmx+1)^3 x nv; mbounds = {mb11, mb12, mb21, mb22,
 * mb31, mb32}. */
void orc_interpolate3d(const int* mx, int nv, const int* mbounds, const int* mthbc,
                       int ipass, double* qf, const int* pmx, const double* qc);

/* Resolved minimum level for the parameters (lib/bsamroutines.f90:287-301). */
int orc_minlevel(const orc_params* p);

/* ---- leaf routines, for known-answer and fixture tests ---------------- */
/* RelaxGrid2D/3D (problem.f90:164-215, 453-518): one colour pass in place.
 * q: (0:mx+1)^d x 2, f: (1:mx)^d x 2.                                   */
void orc_relax_grid(int ndims, const int* mx, double h, double dt,
                    double alpha, double eps, int ipass, double* q,
                    const double* f);
/* Operator2D/3D (problem.f90:231-257, 534-561): res (1:mx)^d x 2.       */
void orc_operator(int ndims, const int* mx, double h, double dt,
                  double alpha, double eps, const double* q, double* res);
/* Restriction2D/3D (gridutilities.f90:89-110, 406-433) of a (1:mx)^d x nv
 * array into (1:mx/2)^d x nv.                                           */
void orc_restriction(int ndims, const int* mx, int nv, const double* a,
                     double* out);
/* BiLin/TriLinProlongationP1 (gridutilities.f90:137-175, 474-529):
 * a (0:cmx+1)^d x nv -> out (0:2cmx+1)^d x nv.                          */
void orc_prolongation_p1(int ndims, const int* cmx, int nv, const double* a,
                         double* out);
/* SetBC2D/3D (boundary.f90:643-891) with the problem's UserBC2D/3D
 * (problem.f90:646-756) on q (0:mx+1)^d x nv, in place.                 */
int orc_setbc(int ndims, const int* mx, int nv, const int* mthbc, double* q);
/* Source2D/3D (problem.f90:258-280, 562-585): f from qold.               */
void orc_source(int ndims, const int* mx, double alpha, const double* qold,
                double* f);
/* ---- regridding leaves -------------------------------------------------- */
/* SetErrFlagsUser2D/3D (problem.f90:135-163, 425-452): flags (1:mx)^d of c
 * (0:mx+1)^d where the undivided central gradient exceeds tol.            */
void orc_errflags(int ndims, const int* mx, double tol, const double* c, int* flags);
/* Bi/TriLinProlongationP1MC (gridutilities.f90:219-279, 588-686):
 * a (0:cmx+1)^d x nv -> out (0:2cmx+1)^d x nv.                          */
void orc_prolong_mc(int ndims, const int* cmx, int nv, const double* a, double* out);
/* NewSubGrids (lib/bsamroutines.f90:1352-1528): Berger-Rigoutsos boxes
 * (lo, hi per dimension; 6 ints each) of flags (1:mx)^d, in the order the
 * reference makes the grids.  Returns the count, -1 if above maxboxes.     */
int orc_new_subgrids(int ndims, const int* mx, const int* flags, double desfill, int mgp,
                     int* boxes, int maxboxes);

/* Energy2D (problem.f90:330-361) of c (0:mx+1)^2.                        */
double orc_energy2d(const int* mx, double h, double alpha, double eps,
                    const double* c);

#ifdef __cplusplus
}
#endif
#endif
