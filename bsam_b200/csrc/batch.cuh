// batch.cuh -- kernels of the batched engine (bsam_batch.cu).
//
// Every V-cycle stage of a tick is one launch over a device-resident work
// list that covers that stage for all resident problems; the list's length
// is read on the device, so problems can be added between ticks without
// re-capturing the tick graph.  CTAs walk the list in runs of consecutive
// tiles (TileRuns) and run the same tile bodies as the single-problem
// kernels (kernels.cuh, mixed.cuh, bottom.cuh); tiles of finished problems
// are skipped.
//
// Per-problem control (k_batch_control) replaces the host loop of
// MultigridIterations (afas:69-104) and of TakeTimeSteps
// (lib/bsamroutines.f90:632-762) for each slot: it sums the slot's own
// residual partials in the same order as last_block_total, so every
// decision matches the single-problem engine bit for bit.
#pragma once
#include "amr.cuh"
#include "bottom.cuh"
#include "kernels.cuh"
#include "mixed.cuh"

namespace bsam {

// SLOT_REGRID: a refined hierarchy between two time steps, waiting for the
// host to regrid it (bsam_batch_submit_amr); its records are inactive.
enum : int32_t {
  SLOT_IDLE = 0,
  SLOT_RUNNING = 1,
  SLOT_DONE = 2,
  SLOT_FAILED = 3,
  SLOT_REGRID = 4
};

// Slot kinds (SlotCfg::kind).
enum : int32_t { SLOT_UNIFORM = 0, SLOT_AMR = 1 };

// Host-owned per-slot configuration (rewritten whenever lists are rebuilt).
struct SlotCfg {
  int32_t ib, ie;     // the slot's tiles in the master list (its residual partials)
  int32_t rec0, nrec; // its patch records
  int32_t master;     // record holding the FP64 state
  int32_t nsteps, maxv;
  int32_t kind;       // SLOT_UNIFORM: records in the batch's table, partials of
                      // the master list; SLOT_AMR: records in the refined
                      // hierarchies' table, partials of their master list
  double denom;       // nrvars * cells (L2Error's integralresult(2))
  double tol;
};

// The streaming kernels over tile lists are bound by memory latency.  For the
// FP64 defect, the FP64 update and the 2D correction a register cap of 48
// (ten 128-thread CTAs per SM) puts more loads in flight and measured 11-17 %
// faster; restriction and coarse load measured slower under that cap (the
// coarse load takes a cap of 64 instead).
constexpr int BATCH_LATENCY_MIN_BLOCKS = 10;

// Device-owned per-slot state (the host writes it only at admission).
struct SlotState {
  int32_t phase, step, iters, vcycles;
};

struct StepLog {
  int32_t nv, conv;
  double res;
};

// Mirror in mapped host memory: what the host polls.
struct SlotOut {
  int32_t phase, step, vcycles, pad_;
};

struct BatchCtl {
  int32_t ticks_left;  // ticks this graph launch may still run
  int32_t running;     // slots still running after this tick's control pass
  int32_t kerr;        // nonzero: a fused stage's copy wait gave up (fused2.cuh)
  int32_t pad_;
  int64_t ticks;       // ticks executed since creation
};

template <class T, int D>
__global__ void __launch_bounds__(BLOCK_THREADS)
    kb_relax(const DevPatch* __restrict__ PT, const Item* __restrict__ items,
             const int* __restrict__ count, int color, TileRuns R) {
  const int n = *count;
  for (int b = R.first(); b < n; b = R.next(b)) relax_item<T, D>(PT, items[b], color);
}

// Transfers between a depth-d record (value type TC) and its parent, whose
// type is the record's pprec.
template <class TC, int D>
__global__ void __launch_bounds__(BLOCK_THREADS)
    kb_restrict(const DevPatch* __restrict__ PT, const Item* __restrict__ items,
                const int* __restrict__ count, TileRuns R) {
  const int n = *count;
  for (int b = R.first(); b < n; b = R.next(b)) {
    const Item it = items[b];
    if (PT[it.patch].pprec == PREC_F32) restrict_item<TC, float, D>(PT, it);
    else restrict_item<TC, double, D>(PT, it);
  }
}

// Eight CTAs per SM (a 64-register cap): 1.4 % faster per batch solve than
// the compiler's 80 registers at six, despite a few spilled values.
template <class TC, int D>
__global__ void __launch_bounds__(BLOCK_THREADS, 8)
    kb_coarse_load(const DevPatch* __restrict__ PT, const Item* __restrict__ items,
                   const int* __restrict__ count, TileRuns R) {
  const int n = *count;
  for (int b = R.first(); b < n; b = R.next(b)) {
    const Item it = items[b];
    if (PT[it.patch].pprec == PREC_F32) coarse_load_item<TC, float, D>(PT, it);
    else coarse_load_item<TC, double, D>(PT, it);
  }
}

template <class TC, int D>
__global__ void __launch_bounds__(BLOCK_THREADS)
    kb_correct(const DevPatch* __restrict__ PT, const Item* __restrict__ items,
               const int* __restrict__ count, TileRuns R) {
  const int n = *count;
  for (int b = R.first(); b < n; b = R.next(b)) {
    const Item it = items[b];
    if (PT[it.patch].pprec == PREC_F32) correct_item<TC, float, D>(PT, it);
    else correct_item<TC, double, D>(PT, it);
  }
}

// CorrectFine in 2D by 2 x 2 blocks of fine cells: the fine cells 2m, 2m+1
// (x) and 2n, 2n+1 (y) read the same four parent corrections, formed once
// here; each cell then takes correct_cell's bilinear expression on them, so
// the values are correct_cell's bit for bit.  Block (m, n) for
// m = 0..cn0, n = 0..cn1 covers fine cells 1..n0 x 1..n1 exactly once.
template <class TC, class TP>
__device__ __forceinline__ void correct_block2(const DevPatch& C, const DevPatch& P, int m,
                                               int n) {
  TC* q0 = fld<TC>(mid_state(C)[0]);
  TC* q1 = fld<TC>(mid_state(C)[1]);
  TP e[2][2][2];  // [component][m + a][n + b]
#pragma unroll
  for (int v = 0; v < 2; ++v) {
    const TP* pq = fld<TP>(P.q[v]);
    const TP* ps = fld<TP>(P.qs[v]);
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int bb = 0; bb < 2; ++bb) {
        const int64_t x = cidx(P, C.off[0] + m + a, C.off[1] + n + bb, 0);
        e[v][a][bb] = pq[x] - ps[x];
      }
  }
#pragma unroll
  for (int dy = 0; dy < 2; ++dy) {
    const int J = 2 * n + dy;
    if (J < 1 || J > C.n[1]) continue;
    const bool ey = dy == 0;
#pragma unroll
    for (int dx = 0; dx < 2; ++dx) {
      const int I = 2 * m + dx;
      if (I < 1 || I > C.n[0]) continue;
      const bool ex = dx == 0;
      TP corr[2];
#pragma unroll
      for (int v = 0; v < 2; ++v) {
        const TP b0 = lin_x<TP>(ex, e[v][0][0], e[v][1][0]);
        const TP b1 = lin_x<TP>(ex, e[v][0][1], e[v][1][1]);
        corr[v] = lin_x<TP>(ey, b0, b1) / TP(16);
      }
      const int64_t c = cidx(C, I, J, 0);
      const TC a0 = q0[c] + TC(corr[0]);
      const TC a1 = q1[c] + TC(corr[1]);
      q0[c] = a0;
      q1[c] = a1;
      if (C.wt && near_boundary(C, I, J, 0, 2)) write_through<TC, 2>(C, q0, q1, I, J, 0, a0, a1);
    }
  }
}

// Items: tiles of 32 x TILE_Y blocks (m, n) of a record (list L_CORR).
template <class TC>
__global__ void __launch_bounds__(BLOCK_THREADS, BATCH_LATENCY_MIN_BLOCKS)
    kb_correct2(const DevPatch* __restrict__ PT, const Item* __restrict__ items,
                const int* __restrict__ count, TileRuns R) {
  const int n = *count;
  for (int b = R.first(); b < n; b = R.next(b)) {
    const Item it = items[b];
    const DevPatch C = PT[it.patch];
    if (!C.active) continue;
    const int m = it.tx * 32 + threadIdx.x, nn = it.ty * TILE_Y + threadIdx.y;
    if (m > C.cn[0] || nn > C.cn[1]) continue;
    const DevPatch P = PT[C.parent];
    if (C.pprec == PREC_F32) correct_block2<TC, float>(C, P, m, nn);
    else correct_block2<TC, double>(C, P, m, nn);
  }
}

// Bottom chains (FP64 in both forms), one CTA per chain at a time.  256
// threads at up to 64 registers: four chains per SM run at once, so a batch
// of a few hundred problems has all its chains resident in one wave (cell
// updates within a phase are independent, so the thread count does not
// change any result).
constexpr int BATCH_BOTTOM_THREADS = 256;

template <int D>
__global__ void __launch_bounds__(BATCH_BOTTOM_THREADS, 4)
    kb_bottom(const DevPatch* __restrict__ PT, const Item* __restrict__ tops,
              const int* __restrict__ count, int nu) {
  __shared__ int chain[BOTTOM_MAX_DEPTH];
  __shared__ int depth;
  const int n = *count;
  for (int b = blockIdx.x; b < n; b += gridDim.x) {
    const int top = tops[b].patch;
    if (!PT[top].active) continue;  // uniform per CTA
    bottom_chain<double, D>(PT, top, nu, chain, depth);
  }
}

// Source of the masters whose new time step starts in this tick.
template <int D>
__global__ void __launch_bounds__(BLOCK_THREADS)
    kb_source(const DevPatch* __restrict__ PT, const Item* __restrict__ items,
              const int* __restrict__ count, TileRuns R) {
  const int n = *count;
  for (int b = R.first(); b < n; b = R.next(b)) source_item<double, D>(PT, items[b], 1);
}

// FP64 form: residual partial of every master tile.
template <int D>
__global__ void __launch_bounds__(BLOCK_THREADS)
    kb_resid(const DevPatch* __restrict__ PT, const Item* __restrict__ items,
             const int* __restrict__ count, double* __restrict__ partials, TileRuns R) {
  const int n = *count;
  for (int b = R.first(); b < n; b = R.next(b)) {
    const Item it = items[b];
    const DevPatch P = PT[it.patch];
    if (!P.active) continue;  // uniform per CTA
    const double s = block_sum(resid_item<double, D>(P, it));
    if (threadIdx.x == 0 && threadIdx.y == 0) partials[b] = s;
  }
}

// Mixed form: defect of every master tile (newstep_only = 0, with partials)
// or of the masters starting a time step (newstep_only = 1: twin set-up only).
template <int D>
__global__ void __launch_bounds__(BLOCK_THREADS, BATCH_LATENCY_MIN_BLOCKS)
    kb_defect(const DevPatch* __restrict__ PT, const Item* __restrict__ items,
              const int* __restrict__ count, double* __restrict__ partials, int newstep_only,
              TileRuns R) {
  const int n = *count;
  for (int b = R.first(); b < n; b = R.next(b)) {
    const Item it = items[b];
    const DevPatch M = PT[it.patch];
    if (!M.active || (newstep_only && !M.newstep)) continue;  // uniform per CTA
    const bool w32 = PT[M.twin].prec == PREC_F32;
    const double acc = w32 ? defect_item<float, D>(PT, it, newstep_only)
                           : defect_item<double, D>(PT, it, newstep_only);
    const double s = block_sum(acc);
    if (!newstep_only && threadIdx.x == 0 && threadIdx.y == 0) partials[b] = s;
  }
}

template <int D>
__global__ void __launch_bounds__(BLOCK_THREADS, BATCH_LATENCY_MIN_BLOCKS)
    kb_update(const DevPatch* __restrict__ PT, const Item* __restrict__ items,
              const int* __restrict__ count, TileRuns R) {
  const int n = *count;
  for (int b = R.first(); b < n; b = R.next(b)) {
    const Item it = items[b];
    const DevPatch M = PT[it.patch];
    if (!M.active) continue;
    const DevPatch& W = PT[M.twin];
    if (W.fused) continue;  // updated by its post-smoothing stage (kb_smooth2, upd)
    if (W.prec == PREC_F32) update_item<float, D>(PT, it);
    else update_item<double, D>(PT, it);
  }
}

// ---- refined hierarchies (SLOT_AMR) ---------------------------------------------
//
// The V-cycle of a refined hierarchy runs the single-problem engine's
// per-level kernels as list kernels over the records of every such problem
// at one depth: colour passes (kb_relax), SetGhost of refined levels
// (kb_ghost), restriction, the snapshot of partly covered parents (kb_snap),
// coarse load, correction, FillDown (kb_filldown), all FP64.

// SetGhost(level, ipass) of refined records, a CTA per record at a time:
// items[b] = {record, first transfer, transfer count} into cps.
template <int D>
__global__ void __launch_bounds__(D == 2 ? 128 : 256, D == 2 ? 8 : 4)
    kb_ghost(const DevPatch* __restrict__ PT, const Item* __restrict__ items,
             const int* __restrict__ count, const OverlapCopy* __restrict__ cps, int ipass) {
  const int n = *count;
  for (int b = blockIdx.x; b < n; b += gridDim.x) {
    const Item it = items[b];
    if (!PT[it.patch].active) continue;  // uniform per CTA
    if (D == 2) ghost2_patch(PT, it.patch, cps, make_int2(it.tx, it.ty), ipass);
    else ghost3_patch(PT, it.patch, cps, make_int2(it.tx, it.ty), ipass);
  }
}

// One colour pass (RelaxGrid2D + write-through) over tiles shaped to narrow
// patches: refined patches are 8-64 cells wide, so the 64-column tiles of
// kb_relax leave most lanes idle.  items[b] = {record, tile x, tile y, W}:
// W lanes per row (8, 16 or 32) each take a column pair, 128 / W rows per
// tile; the cell of the pass's colour in each pair is updated as relax_item
// updates it, so the pass is the same whatever the tile shape.
__global__ void __launch_bounds__(BLOCK_THREADS)
    kb_relax_narrow2(const DevPatch* __restrict__ PT, const Item* __restrict__ items,
                     const int* __restrict__ count, int color, TileRuns R) {
  const int n = *count;
  const int t = threadIdx.x + blockDim.x * threadIdx.y;
  for (int b = R.first(); b < n; b = R.next(b)) {
    const Item it = items[b];
    const DevPatch P = PT[it.patch];
    if (!P.active) continue;  // uniform per CTA
    const int W = it.tz;
    const int j = it.ty * (BLOCK_THREADS / W) + t / W + 1;
    if (j > P.n[1]) continue;
    const int i0 = (it.tx * W + t % W) * 2 + 1;
    const int i = i0 + ((i0 + j + color) & 1);
    if (i > P.n[0]) continue;
    relax_cell<double, 2>(P, i, j, 0);
  }
}

// GetCoarseGhostPoints' source for the children of a partly covered parent:
// qs = q over the parent's interior and ring, one row (j, k) per item.
template <int D>
__global__ void __launch_bounds__(BLOCK_THREADS)
    kb_snap(const DevPatch* __restrict__ PT, const Item* __restrict__ items,
            const int* __restrict__ count) {
  const int n = *count;
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int nt = blockDim.x * blockDim.y;
  for (int b = blockIdx.x; b < n; b += gridDim.x) {
    const Item it = items[b];
    const DevPatch P = PT[it.patch];
    if (!P.active) continue;
    for (int i = tid; i < P.n[0] + 2; i += nt) {
      const int64_t c = cidx(P, i, it.ty, D == 3 ? it.tz : 0);
#pragma unroll
      for (int v = 0; v < 2; ++v) fld<double>(P.qs[v])[c] = fld<double>(P.q[v])[c];
    }
  }
}

// FillDownLevel for the solution over footprint tiles of refined records
// (k_filldown's tile body).
template <int D>
__global__ void __launch_bounds__(BLOCK_THREADS)
    kb_filldown(const DevPatch* __restrict__ PT, const Item* __restrict__ items,
                const int* __restrict__ count, TileRuns R) {
  const int n = *count;
  for (int b = R.first(); b < n; b = R.next(b)) {
    const Item it = items[b];
    if (!PT[it.patch].active) continue;
    filldown_item<D>(PT, it);
  }
}

// End of a tick, one CTA per slot: ErrorAFAS of the slot from its partials,
// then MultigridIterations' exit test and TakeTimeSteps' step advance.
// Block of BLOCK_THREADS threads: the partial sums are added in the order of
// last_block_total over the slot's own tiles.
// Refined hierarchies (SLOT_AMR) keep their records in APT and their
// partials in apartials; at the end of a time step that is not their last
// they pause in SLOT_REGRID (records inactive) until the host has regridded
// them and started the next step.
__global__ void __launch_bounds__(BLOCK_THREADS)
    k_batch_control(DevPatch* __restrict__ PT, DevPatch* __restrict__ APT,
                    const SlotCfg* __restrict__ cfg, SlotState* __restrict__ state,
                    StepLog* __restrict__ log, int max_steps, SlotOut* __restrict__ out,
                    const double* __restrict__ partials, const double* __restrict__ apartials,
                    BatchCtl* __restrict__ ctl, int nslots) {
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int nthreads = blockDim.x * blockDim.y;
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    if (state[s].phase != SLOT_RUNNING) continue;  // uniform per CTA
    const SlotCfg C = cfg[s];
    const bool amr = C.kind == SLOT_AMR;
    DevPatch* T = amr ? APT : PT;
    const double* part = amr ? apartials : partials;
    double acc = 0.0;
    for (int b = tid; b < C.ie - C.ib; b += nthreads) acc += part[C.ib + b];
    const double total = block_sum(acc);
    if (tid == 0) {
      SlotState S = state[s];
      const double r = sqrt(total / C.denom);
      S.iters += 1;
      S.vcycles += 1;
      const bool conv = r < C.tol;
      const bool finite = isfinite(r);
      if (!amr) PT[C.master].newstep = 0;
      if (conv || S.iters >= C.maxv || !finite) {
        if (S.step < max_steps) {
          StepLog L;
          L.nv = S.iters;
          L.conv = conv ? 1 : 0;
          L.res = r;
          log[(int64_t)s * max_steps + S.step] = L;
        }
        S.step += 1;
        S.iters = 0;
        if (!finite || S.step >= C.nsteps) {
          S.phase = finite ? SLOT_DONE : SLOT_FAILED;
          for (int r2 = C.rec0; r2 < C.rec0 + C.nrec; ++r2) T[r2].active = 0;
        } else if (amr) {
          S.phase = SLOT_REGRID;  // AMR(rootlevel) on the host, then the next step
          for (int r2 = C.rec0; r2 < C.rec0 + C.nrec; ++r2) T[r2].active = 0;
        } else {
          PT[C.master].newstep = 1;  // CopyQToQold + source at the next tick
        }
      }
      state[s] = S;
      if (S.phase == SLOT_RUNNING) atomicAdd(&ctl->running, 1);
      // Mapped host mirror: counters first, the phase last.
      volatile SlotOut* vo = out + s;
      vo->vcycles = S.vcycles;
      vo->step = S.step;
      __threadfence_system();
      vo->phase = S.phase;
    }
  }
}

// WHILE condition of the tick graph: another tick while some slot runs and
// the launch's tick budget lasts.  in_graph = 0: eager ticks (counters only).
__global__ void k_batch_cond(BatchCtl* __restrict__ ctl, cudaGraphConditionalHandle handle,
                             int in_graph) {
  ctl->ticks += 1;
  const int left = ctl->ticks_left - 1;
  ctl->ticks_left = left;
  const bool again = ctl->running > 0 && left > 0 && ctl->kerr == 0;
  ctl->running = 0;
  if (in_graph) cudaGraphSetConditional(handle, again ? 1u : 0u);
}

// ---- seeded initial state on the device ---------------------------------------
//
// QInit replacement for generated workloads (the reference's QInit2D/3D,
// problem.f90:58-101, 362-397, fills q on the host; here the state of a
// submitted problem can instead be drawn where it lives):
//   c(i,j[,k]) = cbar + amp * U(-1, 1), U from SplitMix64 stream `seed` in
//   column-major interior order, U(a,b) = a + (b - a) * ((x >> 11) * 2^-53);
//   mu = Dfc(c) - Dfe(c) - eps^2/h^2 * ULap(c) with Neumann (copy) ghosts.
// The same arithmetic in the same order as the host generator
// (bsam_b200/workloads.py: uniform, initial_q), so both give identical bits.

__device__ __forceinline__ double seeded_u(uint64_t seed, int64_t idx) {
  uint64_t z = seed + (uint64_t)(idx + 1) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z = z ^ (z >> 31);
  const double u = (double)(z >> 11) * 0x1.0p-53;
  return -1.0 + 2.0 * u;
}

// c at interior-or-ghost cell (i,j,k) under Neumann copy ghosts.
template <int D>
__device__ __forceinline__ double seeded_c(const DevPatch& P, uint64_t seed, double cbar,
                                           double amp, int i, int j, int k) {
  i = i < 1 ? 1 : (i > P.n[0] ? P.n[0] : i);
  j = j < 1 ? 1 : (j > P.n[1] ? P.n[1] : j);
  if (D == 3) k = k < 1 ? 1 : (k > P.n[2] ? P.n[2] : k);
  const int64_t idx = (int64_t)(i - 1) + (int64_t)P.n[0] * ((j - 1) + (int64_t)P.n[1] * (D == 3 ? k - 1 : 0));
  return cbar + amp * seeded_u(seed, idx);
}

// Interior of the state record `rec`: c and mu (ghosts by a k_setbc launch).
template <int D>
__device__ __forceinline__ void init_seeded_range(const DevPatch& P, uint64_t seed, double cbar,
                                                  double amp, double k2, int64_t g0,
                                                  int64_t gstep) {
  const int64_t n = (int64_t)P.n[0] * P.n[1] * (D == 3 ? P.n[2] : 1);
  for (int64_t g = g0; g < n; g += gstep) {
    const int i = (int)(g % P.n[0]) + 1;
    const int64_t r = g / P.n[0];
    const int j = (int)(r % P.n[1]) + 1;
    const int k = D == 3 ? (int)(r / P.n[1]) + 1 : 0;
    const double c = seeded_c<D>(P, seed, cbar, amp, i, j, k);
    // lap = -2d c + (c(i+1) + c(i-1)) + (c(j+1) + c(j-1)) [+ ...], summed
    // left to right per dimension as the host generator does.
    double lap = -2.0 * D * c;
    lap = lap + seeded_c<D>(P, seed, cbar, amp, i + 1, j, k);
    lap = lap + seeded_c<D>(P, seed, cbar, amp, i - 1, j, k);
    lap = lap + seeded_c<D>(P, seed, cbar, amp, i, j + 1, k);
    lap = lap + seeded_c<D>(P, seed, cbar, amp, i, j - 1, k);
    if (D == 3) {
      lap = lap + seeded_c<D>(P, seed, cbar, amp, i, j, k + 1);
      lap = lap + seeded_c<D>(P, seed, cbar, amp, i, j, k - 1);
    }
    const double alpha = P.alpha;
    const double mu = Problem::Dfc(c, alpha) - Problem::Dfe(c, alpha) - k2 * lap;
    const int64_t ci = cidx(P, i, j, k);
    fld<double>(P.q[0])[ci] = c;
    fld<double>(P.q[1])[ci] = mu;
  }
}

template <int D>
__global__ void k_init_seeded(const DevPatch* __restrict__ PT, int rec, uint64_t seed,
                              double cbar, double amp, double k2) {
  const DevPatch P = PT[rec];
  init_seeded_range<D>(P, seed, cbar, amp, k2, (int64_t)blockIdx.x * blockDim.x + threadIdx.x,
                       (int64_t)gridDim.x * blockDim.x);
}

// ---- batched admission ---------------------------------------------------------
//
// Admitting many problems at once (bsam_batch_submit_many) stages their
// patch records, tensor maps and slot states in page-locked host memory and
// lets one launch scatter them (the device reads the host memory directly),
// zeroes their pool regions in one launch and draws their seeded initial
// states in one launch, instead of a few API calls per problem.

// n 8-byte words from src to dst (either side may be page-locked host memory).
struct WordSpan {
  const uint64_t* src;
  uint64_t* dst;
  int64_t n;
};

__global__ void __launch_bounds__(256) k_word_spans(const WordSpan* __restrict__ spans) {
  const WordSpan sp = spans[blockIdx.y];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < sp.n;
       i += (int64_t)gridDim.x * blockDim.x)
    sp.dst[i] = sp.src[i];
}

struct ZeroSpan {
  uint64_t* dst;
  int64_t n;
};

__global__ void __launch_bounds__(256) k_zero_spans(const ZeroSpan* __restrict__ spans) {
  const ZeroSpan sp = spans[blockIdx.y];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < sp.n;
       i += (int64_t)gridDim.x * blockDim.x)
    sp.dst[i] = 0ull;
}

// The seeded initial state of one admitted problem (k_init_seeded's
// arguments).
struct SeedTask {
  int32_t rec, pad_;
  uint64_t seed;
  double cbar, amp, k2;
};

template <int D>
__global__ void k_init_seeded_list(const DevPatch* __restrict__ PT,
                                   const SeedTask* __restrict__ tasks) {
  const SeedTask t = tasks[blockIdx.y];
  const DevPatch P = PT[t.rec];
  init_seeded_range<D>(P, t.seed, t.cbar, t.amp, t.k2,
                       (int64_t)blockIdx.x * blockDim.x + threadIdx.x,
                       (int64_t)gridDim.x * blockDim.x);
}

// One problem's root state between the caller's Fortran-ordered q (both
// components, ghosts included: `rows` rows of e0 values per component) and
// the pitched master fields q0, q1 (row pitch sy; in 3D the plane pitch is
// sy * (n1 + 2), so the rows of every plane follow each other at pitch sy).
// The packed copy lives in the engine's device transfer buffer, which one
// contiguous DMA per problem fills from, or empties into, the caller's
// buffer: pitched host copies of rows this short run far below the link's
// speed.
struct RowsTask {
  double* packed;
  double* q[2];
  int64_t rows, sy;
  int32_t e0, pad_;
};

// A warp per row: packed -> pitched (unpack) or pitched -> packed (pack).
template <bool UNPACK>
__global__ void __launch_bounds__(256) k_rows_list(const RowsTask* __restrict__ tasks) {
  const RowsTask t = tasks[blockIdx.y];
  const int lane = threadIdx.x & 31;
  const int64_t wpb = blockDim.x >> 5;
  for (int64_t r = (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5); r < 2 * t.rows;
       r += (int64_t)gridDim.x * wpb) {
    const int c = r >= t.rows ? 1 : 0;
    double* pitched = t.q[c] + (r - c * t.rows) * t.sy;
    double* packed = t.packed + r * t.e0;
    for (int i = lane; i < t.e0; i += 32) {
      if (UNPACK) pitched[i] = packed[i];
      else packed[i] = pitched[i];
    }
  }
}

__global__ void k_batch_budget(BatchCtl* __restrict__ ctl, int ticks) {
  ctl->ticks_left = ticks;
  ctl->running = 0;
}

}  // namespace bsam
