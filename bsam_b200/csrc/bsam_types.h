// bsam_types.h -- device-resident patch table shared by host and kernels.
//
// Every grid of the hierarchy (root, below-root multigrid levels, AMR
// patches, and the patches of many independent problems in a batch) is one
// DevPatch.  Kernels never loop over levels or problems on the host side of
// the launch: they take a work list of Items (patch, tile) so that one launch
// covers every patch of a level -- or of a V-cycle stage across a batch.
#pragma once
#include <stdint.h>

namespace bsam {

// Tile of cells one CTA handles: 32 threads x 2 cells in x, TILE_Y rows,
// one z plane.  Blocks are (32, TILE_Y).
constexpr int TILE_X = 64;
constexpr int TILE_Y = 4;
constexpr int BLOCK_THREADS = 32 * TILE_Y;

// Per-face ghost rule applied by SetBC (boundary.f90:643-891):
//   BC_NONE    ghost not written by SetBC (internal 999 faces)
//   BC_COPY    q(ghost) = q(mirror)            (mthbc 1; UserBC2D faces 3,4)
//   BC_REFLECT q(ghost) = 2 - q(mirror)        (UserBC2D faces 1,2; UserBC3D)
//   BC_NEGATE  e(ghost) = -e(mirror): BC_REFLECT seen by a correction e of a
//              state q (q = base + e and both obey 2 - q), used by the
//              correction-form levels of the mixed precision cycle
//   BC_PERIODIC (mthbc 2 on both faces of a dimension; PeriodicBC,
//              boundary.f90:417-483, with qpo = 0): the low ghost takes the
//              patch's last interior layer, the high ghost its first
enum : int32_t { BC_NONE = 0, BC_COPY = 1, BC_REFLECT = 2, BC_NEGATE = 3, BC_PERIODIC = 4 };

enum : int32_t { PREC_F64 = 0, PREC_F32 = 1 };

struct DevPatch {
  int32_t ndims;
  int32_t n[3];       // interior cells per dimension (n[2] = 1 in 2D)
  int32_t cn[3];      // this patch's footprint in its parent: n / 2
  int32_t off[3];     // mbounds(:,1) - 1: origin of the footprint in the parent
  int32_t bc[6];      // BC_* per face (x-lo, x-hi, y-lo, y-hi, z-lo, z-hi)
  int32_t parent;     // patch index of the parent, -1 on the coarsest level
  int32_t level;
  int32_t wt;         // 1: every face physical or periodic -> kernels write ghosts through
  int32_t prec;       // PREC_*
  int32_t problem;    // problem (batch slot) this patch belongs to
  int32_t fused;      // 1: smoothing stages run the fused kernel (q -> qb -> q)
  int32_t zchunk;     // fused kernel: planes (3D) / rows (2D) per streaming chunk
  int32_t twin;       // mixed form: the working patch of this FP64 master, else -1
  int32_t master;     // mixed form: the FP64 master of this working patch, else -1
  int32_t delta;      // 1: q holds a correction e of the base state bs (mixed.cuh)
  int32_t active;     // 0: every kernel skips this patch (finished or idle batch slot)
  int32_t newstep;    // batch masters: a new time step starts this iteration
  int32_t pprec;      // PREC_* of the parent (transfer kernels pick their types by it)
  int32_t code[6];    // the reference's face codes mthbc (Interpolate3D tests some by value)
  int64_t sy, sz;     // element strides of j and k
  // Base pointers of element (0,0,0), the low ghost corner, per component.
  void* q[2];         // solution (phi, mu), with ghost ring: the state between stages
  void* qb[2];        // second buffer of fused levels: the pre-smoothed state
  void* f[2];         // right-hand side (source / FAS load), interior used
  void* qs[2];        // snapshot of q after restriction (the children's qc)
  void* qo[2];        // qold
  void* bs;           // correction-form levels: phi of the base state
  const void* tmaps;  // fused levels: TMA tensor maps of q0, q1, qb0, qb1, f0, f1, bs
  // Problem constants, all computed on the host in FP64 exactly as the
  // reference does (problem.f90:183-187, 246-248, 472-476).
  double h, dt, eps2, alpha;
  double tmp1;        // dt / h^2
  double tmp2;        // eps2 / h^2
  double tmp3;        // 2d * eps2 / h^2
};

struct Item {
  int32_t patch;
  int32_t tx, ty, tz;  // tile coordinates
};

// Device-side status of a solve (one per problem slot).
struct DevStatus {
  double sumsq;        // last residual sum of squares
  double residual;     // sqrt(sumsq / (nrvars * ncells))
  double mass;
  double esum;         // last Energy2D partial sum (k_energy2)
  uint32_t ticket;     // last-block-done counter of the reductions
  int32_t converged;
  int32_t kerr;        // nonzero: a kernel's bounded wait gave up (see smooth_fused.cuh)
  int32_t iters;       // V-cycles done in the current MultigridIterations call
};

}  // namespace bsam
