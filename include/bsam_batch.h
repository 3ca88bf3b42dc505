/*
 * bsam_batch.h -- many independent Cahn-Hilliard solves on one GPU.
 *
 * The reference advances one problem per process (TakeTimeSteps ->
 * MultigridIterations, lib/bsamroutines.f90:632-762, lib/afasroutines.f90:
 * 38-106).  A batch holds many such problems ("slots") resident in device
 * memory at once and advances all of them together: one "tick" is one FAS
 * V-cycle (AFASVcycle, afas:488-521) of every running problem, issued as one
 * launch per V-cycle stage across the whole batch, followed by each
 * problem's own convergence test (ErrorAFAS, afas:94-101) and, when it
 * converges or reaches maxvcycles, the start of its next time step
 * (CopyQToQold + GetSourceFunction) -- all decided on the device.  Ticks run
 * inside one CUDA graph with a device-side WHILE loop.
 *
 * Per problem the arithmetic is exactly the single-problem library's
 * (bsam_gpu.h) in the same precision form, so a problem's result does not
 * depend on what else is in the batch: results are bitwise identical alone
 * and in any mix, and bitwise identical to bsam_gpu_multigrid_iterations.
 *
 * Continuous batching: problems may be submitted at any time, also while
 * others are being advanced; a submission is admitted when a slot and its
 * device footprint (bsam_batch_footprint) are free in the batch's memory pool
 * and refused with BSAM_ERR_NOMEM otherwise.  Finished problems are read back
 * and their memory released with bsam_batch_collect.
 *
 * No reference counterpart: the reference has no batched or served form.
 */
#ifndef BSAM_BATCH_H
#define BSAM_BATCH_H
#include <stdint.h>
#include "bsam_gpu.h"
#include "bsam_host.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct bsam_batch bsam_batch;

/* Longest time-step record kept per problem. */
#define BSAM_BATCH_MAX_STEPS 256

/* Slot phases (bsam_batch_poll). */
#define BSAM_SLOT_IDLE 0
#define BSAM_SLOT_RUNNING 1
#define BSAM_SLOT_DONE 2
#define BSAM_SLOT_FAILED 3 /* non-finite residual */
#define BSAM_SLOT_REGRID 4 /* refined hierarchy between two time steps, to be
                              regridded at the next bsam_batch_advance */

typedef struct {
  int32_t ndims;            /* 2 or 3: every problem of the batch */
  int32_t precision;        /* BSAM_PREC_FP64 or BSAM_PREC_MIXED */
  int32_t nsmoothingpasses; /* rundata nsmoothingpasses (2) */
  int32_t maxvcycles;       /* per time step */
  int32_t max_slots;        /* problems resident at once */
  int32_t bottom_cells;     /* levels of at most this many cells run in the one-CTA
                               bottom kernel, in FP64 (0 = 1024; at most 4096) */
  int64_t pool_bytes;       /* device memory for problem state; 0 = half of free */
  double qerrortol;
} bsam_batch_params;

/* One problem: a uniform root grid with its below-root levels (the same
 * &griddata subset bsam_host_build_uniform takes) and its own constants. */
typedef struct {
  bsam_host_grid grid;
  int32_t nsteps; /* time steps to take, 1..BSAM_BATCH_MAX_STEPS */
  int32_t pad_;
  double dt, eps, alpha;
} bsam_batch_problem;

/* Per time step of a problem, as MultigridIterations reports it. */
typedef struct {
  int32_t nvcycles;
  int32_t converged;
  double residual;
} bsam_step_result;

/* Execution choices that leave every result bit unchanged (the autotuner's
 * knobs): grid_ctas caps the CTAs of each stage launch (0 = 16 per SM);
 * eager = 1 issues every tick's kernels from the host instead of the
 * graph's device-side loop (then advance runs exactly max_ticks ticks);
 * per_pass = 1 makes problems admitted afterwards smooth with one launch per
 * colour pass instead of the fused shared-memory stage of 2D levels;
 * fused_ctas caps the CTAs of a fused stage launch (0 = 4 per SM);
 * fused_occ picks the fused stage's build: 3 or 4 resident CTAs per SM with
 * one tile buffer each (a register budget of 85 or 64 per thread), or 2: two
 * CTAs per SM with two tile buffers each, the next tile's copies landing
 * while the current one is computed (0 = 4); tile_chunk and fused_chunk
 * set how a launch's CTAs take the tiles of their work list: runs of that
 * many consecutive tiles, run r to CTA r mod the grid (1 = grid-stride;
 * consecutive tiles mostly share their problem's records, which a run then
 * reads from L1), for the small-tile list kernels (0 = 2) and for the fused
 * stages (0 = 1); regrid_threads sets how many host threads run the regrids
 * of refined problems (bsam_batch_submit_amr) that wait at one advance. */
typedef struct {
  int32_t grid_ctas;
  int32_t eager;
  int32_t per_pass;
  int32_t fused_ctas;
  int32_t fused_occ;
  int32_t tile_chunk;
  int32_t fused_chunk;
  int32_t regrid_threads;  /* host threads for the regrids of refined problems
                              that paused together (0 = the host's hardware
                              threads, at most 16) */
} bsam_batch_tuning;

typedef struct {
  int64_t ticks;          /* V-cycle ticks executed */
  int64_t launches;       /* kernel launches issued for those ticks */
  int64_t kernels_per_tick;
  int64_t captures;       /* tick graph (re)captures */
  int64_t pool_used;      /* bytes of the pool held by resident problems */
  int64_t pool_bytes;
  int32_t resident;       /* slots holding a problem */
  int32_t running;
  /* bsam_batch_profile: finest-depth smoothing stages timed with events */
  int64_t smooth_stages;
  double smooth_ms;
  double smooth_bytes;    /* algorithmic bytes of those stages: per cell of
                             the finest working level, the fields each stage
                             must read and write once (the fused 2D stages:
                             state, f, base, the restriction into or the
                             correction from the parent, the FP64 update) */
  /* refined hierarchies (bsam_batch_submit_amr): regrids run between their
     time steps and the host wall-clock seconds spent running them */
  int64_t regrids;
  double regrid_s;
} bsam_batch_stats;

int bsam_batch_create(bsam_batch** b, int device, const bsam_batch_params* p);
int bsam_batch_destroy(bsam_batch* b);
int bsam_batch_set_tuning(bsam_batch* b, const bsam_batch_tuning* t);

/* Device bytes the problem occupies while resident (its admission size). */
int bsam_batch_footprint(bsam_batch* b, const bsam_batch_problem* prob, int64_t* bytes);

/* Admits a problem with initial root state q0 (Fortran layout
 * q(0:mx+1, 0:my+1[, 0:mz+1], 2), ghost values are replaced by SetBC).  The
 * copy is queued behind the work already issued; q0 may be reused on return.
 * *slot receives the problem's slot.  BSAM_ERR_NOMEM: no free slot or not
 * enough pool memory now (retry after a collect). */
int bsam_batch_submit(bsam_batch* b, const bsam_batch_problem* prob, const double* q0,
                      int* slot);

/* As bsam_batch_submit, with the initial state drawn on the device instead of
 * copied (QInit for generated workloads):
 *   c  = cbar + amp * U(-1, 1), U from the SplitMix64 stream `seed` in
 *        column-major interior order (U = -1 + 2 * ((x >> 11) * 2^-53)),
 *   mu = Dfc(c) - Dfe(c) - eps^2/h^2 * ULap(c), Neumann ghosts for ULap;
 * then SetBC.  Bit-identical to building the same q0 on the host. */
int bsam_batch_submit_seeded(bsam_batch* b, const bsam_batch_problem* prob, uint64_t seed,
                             double cbar, double amp, int* slot);

/* Admits problems[0..n) in order, as n calls of bsam_batch_submit would,
 * with their device work batched (a handful of launches for all of them and
 * one pitched copy per component and problem).  Admission stops at the first
 * problem that does not fit now: slots[k] receives the slot of problem k, or
 * -1 for it and every later one.  Returns the number admitted, or an error
 * code (then none is admitted) when a problem is invalid.  q0s[k] as for
 * bsam_batch_submit, except that page-locked q0 buffers are read
 * asynchronously: keep them unchanged until the next call that waits
 * (bsam_batch_sync, bsam_batch_run, a collect).  No reference counterpart. */
int bsam_batch_submit_many(bsam_batch* b, int n, const bsam_batch_problem* problems,
                           const double* const* q0s, int* slots);

/* As bsam_batch_submit_many with the seeded initial state of
 * bsam_batch_submit_seeded (seeds[k], cbar[k], amp[k] for problem k). */
int bsam_batch_submit_seeded_many(bsam_batch* b, int n, const bsam_batch_problem* problems,
                                  const uint64_t* seeds, const double* cbar,
                                  const double* amp, int* slots);

/* Hands the next nsteps time steps of a refined (AMR) hierarchy to the
 * batch: the native driver `a` (bsam_amr_create, FP64 engine on the batch's
 * device, same ndims and nsmoothingpasses) keeps the problem's fields and
 * regrids it before every step (bsam_amr_regrid, at the bsam_batch_advance
 * after the step before ends), and the batch runs each step's
 * MultigridIterations in the launches it issues for all its problems: one
 * launch per V-cycle stage and depth covers the patches of every refined
 * hierarchy resident (colour passes, SetGhost of refined levels,
 * restriction, coarse load, correction, FillDown, ErrorAFAS), so many such
 * problems share the launches that one problem alone leaves latency-bound.
 * The engine's own run parameters (maxvcycles, qerrortol) apply.  Results
 * are bitwise those of nsteps calls of bsam_amr_step.  Until the slot is
 * collected (bsam_batch_collect; collect_many refuses it), the caller must
 * not use the driver or its engine.  Occupies a slot but no pool memory.
 * A regrid that fails ends its problem as BSAM_SLOT_FAILED (the advance that
 * ran it returns the error; the other problems go on).
 * Replaces the time-step loop of TakeTimeSteps (lib/bsamroutines.f90:
 * 632-723) for that problem; no reference counterpart for the batching. */
int bsam_batch_submit_amr(bsam_batch* b, bsam_amr* a, int nsteps, int* slot);

/* 1 while work queued on the batch's stream is still executing, 0 when idle
 * (does not wait). */
int bsam_batch_busy(bsam_batch* b);

/* Queues up to max_ticks V-cycle ticks (fewer if every problem finishes);
 * returns without waiting. */
int bsam_batch_advance(bsam_batch* b, int max_ticks);

/* Waits for all queued work. */
int bsam_batch_sync(bsam_batch* b);

/* Advances until no problem is running (waits). */
int bsam_batch_run(bsam_batch* b);

/* Slots whose problems have finished (DONE or FAILED) and are not yet
 * collected, as seen by the work completed so far (does not wait).  Returns
 * their number; up to maxn are written to slots. */
int bsam_batch_poll(bsam_batch* b, int* slots, int maxn);

/* Phase of a slot as seen by the work completed so far (BSAM_SLOT_*), and
 * the number of time steps it has completed. */
int bsam_batch_slot_phase(bsam_batch* b, int slot, int* phase, int* steps_done);

/* Reads back a finished problem and releases its slot and memory (waits for
 * queued work).  Optional outputs (NULL to skip): root q with ghost ring,
 * one bsam_step_result per time step (nsteps entries), FP64 mass of phi
 * (AfterStep's integral(1)). */
int bsam_batch_collect(bsam_batch* b, int slot, double* q, bsam_step_result* steps,
                       double* mass);

/* bsam_batch_collect of slots[0..n) with one wait: qs[k], steps[k] (arrays
 * of pointers, NULL entries or NULL arrays to skip) and masses[k] (NULL to
 * skip, which saves a reduction per problem).  Every slot must be finished
 * or finish with the work already queued; all are released.  Without masses
 * the call waits only for these slots, not for ticks queued after them
 * (bsam_batch_advance issued before the call keeps the device busy while
 * the results are copied out); with masses it waits for all queued work.
 * BSAM_ERR_DIVERGED when any of them failed.  No reference counterpart. */
int bsam_batch_collect_many(bsam_batch* b, int n, const int* slots, double* const* qs,
                            bsam_step_result* const* steps, double* masses);

/* enable != 0: ticks run eagerly, one at a time, and each finest-depth
 * smoothing stage (2 x nsmoothingpasses colour passes over every running
 * problem's root level; in the mixed 2D form the post-smoothing stage also
 * applies the FP64 update q64 += e) is timed with CUDA events into the
 * stats; 0 stops. */
int bsam_batch_profile(bsam_batch* b, int enable);

int bsam_batch_get_stream(bsam_batch* b, void** stream);
int bsam_batch_get_stats(bsam_batch* b, bsam_batch_stats* s);
const char* bsam_batch_last_error(bsam_batch* b);

#ifdef __cplusplus
}
#endif
#endif
