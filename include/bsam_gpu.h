/*
 * bsam_gpu.h -- C ABI of the B200-native FAS multigrid V-cycle for the BSAM
 * simple_cahn-hilliard problem module.
 *
 * Plain C types only (no CUDA or torch types), callable from Fortran through
 * iso_c_binding (bind(C)) or from C/C++/Python ctypes.  Every call returns an
 * int status: 0 = BSAM_OK (matches err_OK = 0, lib/treeops.f90:66), negative
 * values are errors; bsam_gpu_strerror() names them.  The library never exits
 * or stops the process.
 *
 * Array arguments use the reference's Fortran layout: column-major, i fastest,
 * with the patch's ghost ring for q/qold, q(0:mx1+1, 0:mx2+1[, 0:mx3+1], 1:2)
 * (lib/bsamstorage.f90:74-102), and interior-only f(1:mx1, 1:mx2[, 1:mx3], 1:2).
 * Arrays are copied during the call and never retained.
 */
#ifndef BSAM_GPU_H
#define BSAM_GPU_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum {
  BSAM_OK = 0,
  BSAM_ERR_ARG = -1,        /* invalid argument or parameter */
  BSAM_ERR_CUDA = -2,       /* a CUDA runtime call failed */
  BSAM_ERR_NOMEM = -3,      /* device allocation failed */
  BSAM_ERR_STATE = -4,      /* call out of order (e.g. no hierarchy yet) */
  BSAM_ERR_UNSUPPORTED = -5,/* configuration not supported by this build */
  BSAM_ERR_NODEVICE = -6,   /* no CUDA device / kernels unavailable */
  BSAM_ERR_DIVERGED = -7,   /* non-finite residual detected */
  BSAM_ERR_TOO_LARGE = -8   /* patch exceeds the static scratch of *_noalloc */
};

/* Field selectors for put/get (the nodeinfo components of
 * lib/nodeinfodef.f90:204-215 that the hot path reads or writes). */
enum { BSAM_FIELD_Q = 0, BSAM_FIELD_QOLD = 1, BSAM_FIELD_F = 2 };

/* Precision of the solve. */
enum { BSAM_PREC_FP64 = 0, BSAM_PREC_MIXED = 1 };

typedef struct bsam_gpu bsam_gpu; /* opaque handle: one per host thread */

/* Run parameters: the &rundata / &problemdata values the hot path reads
 * (lib/bsamroutines.f90:68-100; problems/simple_cahn-hilliard/problem.f90:17,
 * problemdef.f90:4).  nrvars must be 2, mbc 1, maux 0, errortype 1. */
typedef struct {
  int32_t ndims, nrvars, mbc, maux;
  int32_t nsmoothingpasses, maxvcycles, errortype, precision;
  double dt, qerrortol, alpha, eps;
} bsam_run_params;

/* One patch of the hierarchy: the nodeinfo geometry (lib/nodeinfodef.f90:
 * 172-207).  Indices follow the Fortran conventions (1-based boxes).
 * parent: index of the parent in the patch array, -1 for the coarsest level.
 * mbounds: this patch's index box in its parent (lib/treeops via
 * InitSeed/MakeNewGrid).  mthbc per face: 1 Neumann reflection, 10-99 the
 * problem's UserBC, 999 internal (coarse-fine), 2 periodic (PeriodicBC; both
 * faces of a dimension, hierarchies without refined levels).  dx is the
 * grid spacing. */
typedef struct {
  int32_t level, parent;
  int32_t mx[3];
  int32_t mbounds[3][2];
  int32_t mglobal[3][2];
  int32_t mthbc[6];
  double dx;
  double xlower[3];
} bsam_patch_desc;

/* Replaces nothing in the reference: creates the device context on CUDA
 * device `device` (one stream per handle). */
int bsam_gpu_create(bsam_gpu** h, int device, const bsam_run_params* p);

/* Kernel-shape choices (no reference counterpart).  Results do not depend on
 * them: every choice computes the same arithmetic in the same order.
 *   fuse_smoother  -1 automatic, 0 one launch per colour pass, 1 fused stage
 *                  (all 2*nu passes of LevelRelax in one launch) where the
 *                  level allows it
 *   fuse_min_n     smallest extent per dimension of a fused level
 *   chunk          planes (3D) / rows (2D) per streaming chunk, 0 = automatic
 *   bottom_cells   levels of at most this many cells run their whole part of
 *                  the V-cycle in one single-CTA launch (at most 4096);
 *                  0 = default (1024 in 2D, 512 in 3D), -1 = never.  In the
 *                  mixed form these levels are FP64; under the default and
 *                  with -1, levels of at most 4096 cells are FP64 (the bits
 *                  do not depend on which of them run in the bottom launch)
 *   graph          0 = run the V-cycle loop of MultigridIterations as one
 *                  captured CUDA graph with a device-side WHILE node (one
 *                  launch per call); -1 = host loop (one launch per kernel,
 *                  one host synchronisation per V-cycle)
 * Call before bsam_gpu_set_hierarchy. */
typedef struct {
  int32_t fuse_smoother;
  int32_t fuse_min_n;
  int32_t chunk;
  int32_t bottom_cells;
  int32_t graph;
  int32_t reserved[3];
} bsam_tuning;
int bsam_gpu_set_tuning(bsam_gpu* h, const bsam_tuning* t);

/* Discrete free energy of the root state, Energy2D (problem.f90:330-361) as
 * AfterStep2D accumulates it into integralresult(2) at level 0
 * (problem.f90:121-123): h^2 (sum Ff(c) + eps^2/h^2/4 sum of the four
 * squared one-sided differences of c per cell), with c = q(:,:,1) and its
 * current ghost ring.  2D hierarchies without refined levels only
 * (BSAM_ERR_UNSUPPORTED otherwise: the reference has no Energy3D).
 * Deterministic; equal to the sequential sums to within rounding. */
int bsam_gpu_energy(bsam_gpu* h, double* energy);

/* ---- regridding on the device ------------------------------------------- */
/* Cell tags of a patch on a level >= 0 for the next regrid, SetErrFlagsUser
 * (problem.f90:135-163, 425-452): flags[cell] = 1 where the undivided central
 * gradient of c = q(...,1) (ghost ring as it stands) exceeds tol, else 0;
 * flags: (1:mx)^d bytes, column-major.  The clustering of the flags into new
 * patches is bsam_host_new_subgrids. */
int bsam_gpu_errflags(bsam_gpu* h, int patch, double tol, uint8_t* flags);

/* InitFields (lib/bsamroutines.f90:1685-1772) of a refined patch of the
 * current hierarchy: q on (0:mx+1)^d becomes the mass-corrected linear
 * prolongation (Bi/TriLinProlongationP1MC, gridutilities.f90:219-279,
 * 588-686) of its parent's q over the patch's footprint and one-cell ring,
 * and qold = q.  TransferValues from an old patch of the same level is a
 * bsam_gpu_put_field of the overlapping cells afterwards.  FP64 form. */
int bsam_gpu_init_patch(bsam_gpu* h, int patch);

/* RestrictSolution of every patch of a refined level into its parent
 * (afas:600-644: parent%q(mbounds) = Restriction(q)), then SetGhost of the
 * parent level: the state changes EstimateLevelErrors makes before tagging
 * the level (lib/bsamroutines.f90:963-1002). */
int bsam_gpu_restrict_level(bsam_gpu* h, int level);

/* SetGhost(level, 0) (boundary.f90:58-89) of one level alone (coarse-fine
 * interpolation, sibling exchange and physical faces above the root; physical
 * faces at and below it), as AMR(level) starts (lib/bsamroutines.f90:939-961). */
int bsam_gpu_set_ghost_level(bsam_gpu* h, int level);

/* Replaces the tree set-up that makes the hierarchy reachable to
 * MultigridIterations: RootInit/InitSeed/AllocFields
 * (lib/bsamroutines.f90:205-494, lib/bsamstorage.f90:46-123).  patches[] is in
 * ApplyOnLevel order within each level (lib/treeops.f90:536-572).  Device
 * fields are allocated and zeroed (AllocFields sets q = qold = 0). */
int bsam_gpu_set_hierarchy(bsam_gpu* h, int npatch, const bsam_patch_desc* patches,
                           int finestlevel);

/* Copy a host field of one patch to the device (BSAM_FIELD_Q/QOLD: array with
 * ghost ring; BSAM_FIELD_F: interior only). */
int bsam_gpu_put_field(bsam_gpu* h, int patch, int field, const double* a);

/* Copy a device field of one patch back to the host, same layouts. */
int bsam_gpu_get_field(bsam_gpu* h, int patch, int field, double* out);

/* SetGhost(level, 0) (lib/boundary.f90:58-89) on every level, coarse to
 * fine, as BSAMSolver does after QInit (lib/bsamroutines.f90:144).  Above the
 * root: coarse-fine interpolation (Interpolate2D), sibling exchange
 * (GhostOverlap) and physical faces. */
int bsam_gpu_set_ghost(bsam_gpu* h);

/* FillDown(solutionfield) (lib/afasroutines.f90:223-310): the refined
 * levels' q restricted into their parents (with the parents' SetGhost), as
 * TakeTimeSteps does on its first step (lib/bsamroutines.f90:651-654).  A
 * no-op without refined levels. */
int bsam_gpu_fill_down(bsam_gpu* h);

/* CopyQToQold on all levels (lib/bsamroutines.f90:568-580, 659-661). */
int bsam_gpu_copy_q_to_qold(bsam_gpu* h);

/* Replaces MultigridIterations (lib/afasroutines.f90:38-106): source set-up
 * followed by up to maxvcycles FAS V(nu,nu) cycles until the finest-level
 * residual (ErrorAFAS, errortype 1) drops below qerrortol.
 *   nvcycles  V-cycles performed
 *   residual  last residual
 *   converged 1 if residual < qerrortol (reference: lconverged), else 0
 * Non-convergence is not an error, as in the reference. */
int bsam_gpu_multigrid_iterations(bsam_gpu* h, int* nvcycles, double* residual,
                                  int* converged);

/* Residuals of each V-cycle of the last multigrid_iterations call (the
 * reference prints them, lib/afasroutines.f90:95).  Returns the count. */
int bsam_gpu_residual_trace(bsam_gpu* h, double* out, int maxn);

/* FP64 mass h^d * sum(phi) over the root level: AfterStep2D/3D integral(1)
 * (problems/simple_cahn-hilliard/problem.f90:121-122, 416-418). */
int bsam_gpu_mass(bsam_gpu* h, double* mass);

/* AfterStepStatistics (lib/bsamroutines.f90:893-937) over the whole
 * hierarchy, finest level first: integral[0] = the composite mass (root
 * h^d sum(c), plus on each refined patch h^d sum(c) - (2h)^d sum(parent c
 * over its footprint)); integral[1] = the composite Energy2D the same way
 * (AfterStep2D, problem.f90:102-134), 0 in 3D (AfterStep3D,
 * problem.f90:398-424 adds none).  FP64 patches only. */
int bsam_gpu_after_step_stats(bsam_gpu* h, double* integral);

/* Regridding with the state resident on the device (FP64 form).
 * bsam_gpu_stash: copy q of every refined patch aside -- the old grids as
 * GridAdapt's TransferValues reads them (lib/bsamroutines.f90:1314-1316);
 * stash index = the patch's index in the table at the time of the call.
 * bsam_gpu_regrid: set the new patch table (as bsam_gpu_set_hierarchy) and
 * fill it on the device: patch i takes q and qold of old patch carry[i]
 * (same level and size) or, with carry[i] = -1 (refined patches only), the
 * mass-corrected prolongation of its parent (InitFields, 1685-1772); then
 * for each pair (new grid, stashed grid) of `transfer` (2 * ntransfer ints)
 * the new grid takes the stashed grid's q on the interior cells both cover
 * (TransferValues / TransferOverlap, 1774-1867). */
/* SetErrFlagsUser of every patch on `level` (table order), the flags of
 * each patch's (1:mx)^d cells concatenated in `flags`: one transfer. */
int bsam_gpu_errflags_level(bsam_gpu* h, int level, double tol, uint8_t* flags);

/* The tagging of every patch of `level` (as bsam_gpu_errflags_level), then
 * its buffering by `ibuffer` cells (BufferAndList + InflateEdgeTags,
 * lib/bsamroutines.f90:1159-1284: the union of every flagged cell's buffer
 * box over the level's patches, as bsam_host_buffer_flags), then per patch
 * the inclusive summed-area table of the buffered flags, all on the device.
 * sat receives the tables of the level's patches in table order, each
 * mx1 * mx2 [* mx3] int32 values, i fastest: sat(i,j,k) = the number of
 * flagged cells in (1:i, 1:j, 1:k).  bsam_host_new_subgrids_sat clusters from
 * them (NewSubGrids' signatures and fill ratios are box counts). */
int bsam_gpu_tag_level(bsam_gpu* h, int level, double tol, int ibuffer, int32_t* sat);
int bsam_gpu_stash(bsam_gpu* h);
int bsam_gpu_regrid(bsam_gpu* h, int npatch, const bsam_patch_desc* patches, int finestlevel,
                    const int* carry, int ntransfer, const int* transfer);

/* The CUDA stream (cudaStream_t) every kernel of this handle runs on, for
 * callers that order their own work or record events against it. */
int bsam_gpu_get_stream(bsam_gpu* h, void** stream);

/* Instrumentation counters since the last bsam_gpu_profile(h, 1) call. */
typedef struct {
  int64_t launches;       /* kernels launched by the library */
  int64_t smooth_stages;  /* timed finest-level smoothing stages (nu sweeps) */
  int64_t smooth_cells;   /* cells per timed stage, summed over stages */
  double smooth_ms;       /* CUDA-event time of those stages */
  double smooth_bytes;    /* algorithmic bytes: 6 * sizeof(value) per cell */
} bsam_gpu_stats;

/* enable = 1: reset the counters and time every finest-level smoothing stage
 * with CUDA events on the handle's stream; 0: stop timing (counters kept). */
int bsam_gpu_profile(bsam_gpu* h, int enable);
int bsam_gpu_get_stats(bsam_gpu* h, bsam_gpu_stats* out);

/* Release the handle and its device memory. */
int bsam_gpu_destroy(bsam_gpu* h);

/* Name of a status code (static string). */
const char* bsam_gpu_strerror(int code);

/* Detail message of the last failing call on this handle (valid until the
 * next call on the handle). */
const char* bsam_gpu_last_error(bsam_gpu* h);

/* Residual norm of one uniform patch, allocating no device memory.
 *
 * No counterpart in the reference.  It is for callers that cannot allocate
 * device memory at the point where they need the norm: a host that has given
 * all device memory to its own pool (a Fortran code's preallocated arena,
 * PyTorch's caching allocator) or a step loop that must not pay the implicit
 * device synchronisation of cudaMalloc/cudaFree.  It returns the same number
 * as the final residual of bsam_gpu_multigrid_iterations (ErrorAFAS with
 * errortype 1, lib/afasroutines.f90:108-221) for fields held by the caller:
 *   q    device pointer, q(0:mx1+1, 0:mx2+1[, 0:mx3+1], 1:2), ghost ring set
 *   f    device pointer, f(1:mx1, 1:mx2[, 1:mx3], 1:2)
 *   out  device pointer to 2 doubles: out[0] = residual, out[1] = sum of rf^2,
 *        written by a kernel on `stream` (NULL = legacy default stream);
 *        synchronise the stream before reading them.
 * Reductions go through one fixed scratch array compiled into the library
 * (about 512 KiB held on every GPU that loads it until the process exits),
 * so the patch may span at most BSAM_NOALLOC_MAX_TILES tiles of 64 x 4 x 1
 * cells (16,777,216 cells when mx1 is a multiple of 64 and mx2 of 4); larger
 * patches return BSAM_ERR_TOO_LARGE.  The first call on a device looks up the
 * scratch array's device address with cudaGetSymbolAddress, so make that
 * first call before capturing any stream.  That address is kept for the life
 * of the process: after a cudaDeviceReset of the device it is stale, so do
 * not call this entry point on a device that was reset.  All calls share the
 * scratch: calls whose kernels overlap on the GPU race and give wrong
 * results. */
#define BSAM_NOALLOC_MAX_TILES 65536
int bsam_gpu_resid_norm_noalloc(int device, int ndims, const int32_t* mx, double dx, double dt,
                                double eps, double alpha, const double* q, const double* f,
                                double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif
