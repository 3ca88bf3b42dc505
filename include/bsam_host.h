/*
 * bsam_host.h -- host driver above the C ABI (bsam_gpu.h).
 *
 * Restates, in C++, the part of the reference's Fortran driver that sets up a
 * uniform root grid with its below-root multigrid levels and advances it in
 * time, calling the C ABI where the Fortran calls MultigridIterations.  A
 * Fortran host would make the same calls through iso_c_binding.
 */
#ifndef BSAM_HOST_H
#define BSAM_HOST_H
#include <stdint.h>
#include "bsam_gpu.h"
#ifdef __cplusplus
extern "C" {
#endif

/* The &griddata values of a single uniform root grid
 * (lib/bsamroutines.f90:219-244; maxlevel = 0). */
typedef struct {
  int32_t ndims;
  int32_t mx[3];
  int32_t mthbc[6];
  int32_t minlevel;  /* <= 0, or 1 for the automatic choice */
  int32_t pad_;
  double xlower[3], xupper[3];
} bsam_host_grid;

/* Number of levels (root + below-root) the grid gets. */
int bsam_host_levels(const bsam_host_grid* g);

/* Replaces RootInit + CreateBelowSeedLevels + InitSeed
 * (lib/bsamroutines.f90:205-494, lib/treeops.f90:193-289): fills out[0] with
 * the root and out[l] with level -l, ready for bsam_gpu_set_hierarchy. */
int bsam_host_build_uniform(const bsam_host_grid* g, bsam_patch_desc* out, int maxn,
                            int* npatch);

/* Replaces the time-step loop of TakeTimeSteps for maxlevel = 0, eqfn = 1
 * (lib/bsamroutines.f90:632-762): per step SetGhost(root,0), CopyQToQold,
 * MultigridIterations.  Optional outputs per step (NULL to skip): root q with
 * ghost ring at q_steps + step*q_stride, V-cycle count, final residual,
 * convergence flag, FP64 mass. */
int bsam_host_take_time_steps(bsam_gpu* h, int nsteps, int root_patch, double* q_steps,
                              int64_t q_stride, int* nvcycles, double* residuals,
                              int* converged, double* mass);

/* Berger-Rigoutsos clustering of a patch's cell flags into new refined
 * patches, as NewSubGrids does it (lib/bsamroutines.f90:1352-1528, with
 * GetSignatures 1530-1554 and GridFlagRatio 1556-1579): starting from the
 * whole patch, each box is trimmed to its flagged rows and columns and, while
 * its flagged fraction is below desfill, split at a hole of the signature
 * (a zero at least mgp cells from both ends) or else at its strongest
 * inflection, keeping every side at least mgp cells.  flags: (1:mx)^d,
 * column-major, nonzero = flagged.  boxes: 6 ints per box (lo, hi in each of
 * three dimensions, 1 beyond ndims) in the order the reference makes the new
 * grids (MakeNewGrid's mbounds).  Returns the number of boxes (0: nothing
 * flagged), BSAM_ERR_ARG for bad arguments or more than maxboxes boxes. */
int bsam_host_new_subgrids(int ndims, const int* mx, const uint8_t* flags, double desfill,
                           int mgp, int* boxes, int maxboxes);

/* bsam_host_new_subgrids from the patch's inclusive summed-area table of its
 * flags (sat(i,j,k) = flagged cells in (1:i, 1:j, 1:k), i fastest, as
 * bsam_gpu_tag_level returns it): every count of a box or a signature slab
 * in constant time; the same boxes in the same order. */
int bsam_host_new_subgrids_sat(int ndims, const int* mx, const int32_t* sat, double desfill,
                               int mgp, int* boxes, int maxboxes);

/* Buffering of the cell flags of one level's patches, as BufferAndList and
 * InflateEdgeTags do it (lib/bsamroutines.f90:1159-1284): every cell flagged
 * before the call flags the cells within ibuffer of it (a cube in global
 * indices) on every patch of the level.  Patch p has mx[3p..3p+2] cells,
 * global index box mglobal[6p..6p+5] (lo, hi per dimension) and flags at
 * flags + offset of the patches before it, (1:mx)^d bytes each; in place. */
int bsam_host_buffer_flags(int ndims, int npatch, const int* mx, const int* mglobal,
                           uint8_t* flags, int ibuffer);

/* The record MakeNewGrid gives the child of `parent` (index parent_index in
 * the caller's table) over the parent box `box` (lo, hi per dimension)
 * (lib/bsamroutines.f90:1581-1683): twice the box's cells, mbounds = box,
 * the global box at the finer level, the parent's physical face codes on the
 * faces the box shares with the parent, 999 elsewhere, xlower of the box's
 * first cell, dx halved. */
int bsam_host_child_desc(int ndims, const bsam_patch_desc* parent, int parent_index,
                         const int* box, bsam_patch_desc* child);

/* WriteQ (lib/bsaminputoutput.f90:51-172): the frame file of a hierarchy --
 * time (f25.12), finestlevel (i3), then per patch on levels 0 .. finestlevel
 * in table order: a blank record, "level ndims 2 nrvars" (i3), dx, xlower,
 * xupper (f25.12), mx, mglobal (i8), and q with its ghost ring, one cell a
 * record, i fastest (2D: es20.12 values, 3D: f25.12; two blanks between).
 * q[p]: patch p's (0:mx+1)^d x 2 array, column-major (ignored, may be NULL,
 * for patches below the root). */
int bsam_host_format_frame(const char* path, int ndims, double time, int finestlevel,
                           int npatch, const bsam_patch_desc* patches, const double* const* q);

/* The frame file of the hierarchy resident in h (patch table `patches`, as
 * given to bsam_gpu_set_hierarchy): q of every patch on a level >= 0 read
 * back with bsam_gpu_get_field, then bsam_host_format_frame. */
int bsam_host_write_frame(bsam_gpu* h, const char* path, int ndims, double time, int npatch,
                          const bsam_patch_desc* patches);

/* Time steps with regridding every step: TakeTimeSteps with AMR(rootlevel)
 * (lib/bsamroutines.f90:632-723, 939-1002, 1299-1350) over an engine handle
 * in the FP64 form.  The &amrdata values, per level 0 .. maxlevel - 1
 * (lib/nodeinfodef.f90:87-103). */
#define BSAM_AMR_MAXLEVEL 8
typedef struct {
  int32_t maxlevel;
  int32_t ibuffer[BSAM_AMR_MAXLEVEL];
  int32_t minimumgridpoints[BSAM_AMR_MAXLEVEL];
  int32_t pad_;
  double qtolerance[BSAM_AMR_MAXLEVEL];
  double desiredfillratios[BSAM_AMR_MAXLEVEL];
} bsam_regrid_params;

typedef struct bsam_amr bsam_amr;

/* The driver of a hierarchy already set on h (bsam_gpu_set_hierarchy with
 * `patches`) whose q the caller has put: SetGhost on every level >= 0 and
 * CopyQToQold, as BSAMSolver leaves them before its first step. */
int bsam_amr_create(bsam_amr** a, bsam_gpu* h, int ndims, const bsam_regrid_params* p,
                    int npatch, const bsam_patch_desc* patches);
/* One time step: AMR(rootlevel) -- per level SetGhost, EstimateLevelErrors'
 * restriction and tagging, buffering, Berger-Rigoutsos per patch,
 * MakeNewGrid, InitFields and TransferValues on the device -- then FillDown
 * on the first step, CopyQToQold and MultigridIterations. */
int bsam_amr_step(bsam_amr* a, int* nvcycles, double* residual, int* converged);
/* The first half of bsam_amr_step: everything before MultigridIterations
 * (AMR(rootlevel), FillDown on the first step, CopyQToQold).  The batched
 * engine calls it between the time steps it runs for the driver
 * (bsam_batch_submit_amr); bsam_amr_step is this call followed by
 * bsam_gpu_multigrid_iterations. */
int bsam_amr_regrid(bsam_amr* a);
/* The current patch table (after the last step's regrid): returns the count
 * and copies up to maxn records into out (out may be NULL). */
int bsam_amr_table(const bsam_amr* a, bsam_patch_desc* out, int maxn);
void bsam_amr_destroy(bsam_amr* a);
/* Host wall-clock seconds spent per phase of bsam_amr_step, summed over
 * the steps so far (each phase ends with the device idle): the stash, the
 * ghost fills and restrictions, tagging and buffering, clustering and the
 * child records, the regrid on the device, and FillDown + CopyQToQold +
 * MultigridIterations.  Returns the number of steps. */
enum {
  BSAM_AMR_PHASE_STASH = 0,
  BSAM_AMR_PHASE_GHOST = 1,
  BSAM_AMR_PHASE_TAG = 2,
  BSAM_AMR_PHASE_CLUSTER = 3,
  BSAM_AMR_PHASE_REGRID = 4,
  BSAM_AMR_PHASE_SOLVE = 5,
  BSAM_AMR_NPHASE = 6
};
int bsam_amr_profile(const bsam_amr* a, double* seconds, int n);

#ifdef __cplusplus
}
#endif
#endif
