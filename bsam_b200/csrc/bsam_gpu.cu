// bsam_gpu.cu -- C ABI of the B200 FAS V-cycle (include/bsam_gpu.h).
//
// Host orchestration of the reference's MultigridIterations / AFASVcycle
// (lib/afasroutines.f90:38-106, 488-547) over the device patch table.  All
// field storage lives in one device arena per handle and stays resident
// across time steps; host arrays cross the bus only in put/get calls.
//
// Device layout of a field (one component of one patch): element (i,j,k),
// i in [0, mx1+1] etc., lives at base + i + j*sy + k*sz.  The allocation
// starts `lead` elements before element (0,0,0) so that every interior row
// (i = 1) begins on a 128-byte boundary; sy is a multiple of 128 bytes.
//
// Patch records: the caller's patches keep their indices.  The FP64 form
// runs the V-cycle on them directly.  The mixed form (mixed.cuh) appends one
// working "twin" per finest-level patch: the caller's finest patch stays the
// FP64 master state (put/get/mass/source/residual), the twin carries the
// FP32 V-cycle; levels above 4096 cells are FP32, smaller ones FP64.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/bsam_gpu.h"
#include "bsam_types.h"
#include "kernels.cuh"
#include "smooth_fused.cuh"
#include "bottom.cuh"
#include "mixed.cuh"
#include "amr.cuh"
#include "regrid.cuh"
#include "stats.cuh"
#include "engine_view.h"

using namespace bsam;

namespace {

// Levels with at most this many cells per patch stay FP64 in the mixed form.
constexpr int64_t MIXED_FP64_CELLS = 4096;
// Default largest level of the one-CTA bottom chain, per dimensionality.
constexpr int DEFAULT_BOTTOM_CELLS_2D = 1024;
constexpr int DEFAULT_BOTTOM_CELLS_3D = 512;

struct LevelPlan {
  int level = 0;
  std::vector<int> patches;  // records the V-cycle runs on (ApplyOnLevel order)
  Item* d_fine = nullptr;    // tiles over each patch's interior
  int nfine = 0;
  Item* d_coarse = nullptr;  // tiles over each patch's footprint in its parent
  int ncoarse = 0;
  Item* d_fused = nullptr;   // fused-stage tiles (tile x, tile y, z chunk)
  int nfused = 0;
  bool fused = false;
  int prec = PREC_F64;
  // AMR levels (above the root): SetGhost is coarse-fine interpolation +
  // sibling exchange + SetBC, over the level's patch list.
  bool amr = false;
  int* d_plist = nullptr;       // the level's patches
  int nplist = 0;
  OverlapCopy* d_ovl = nullptr; // GhostOverlap transfers (ApplyOnLevelPairs order)
  int novl = 0;
  // The same transfers grouped by destination, and per entry of d_plist the
  // {first, count} of its group (the one-launch SetGhost of 2D levels).
  OverlapCopy* d_ovl_by_dst = nullptr;
  int2* d_ovl_range = nullptr;
  // Parent of a refined level: its children do not cover it, so the
  // snapshot qs is a full copy of q taken after restriction + SetGhost.
  bool snap = false;
};

}  // namespace

struct bsam_gpu {
  int device = 0;
  cudaStream_t stream = nullptr;
  bsam_run_params rp{};
  bool have_hierarchy = false;
  bool mixed = false;
  int minlevel = 0, finestlevel = 0;
  int nuser = 0;                     // caller's patches: records [0, nuser)
  std::vector<bsam_patch_desc> desc;
  std::vector<DevPatch> hp;
  std::vector<int64_t> field_elems;  // elements per field allocation, per record
  DevPatch* d_patches = nullptr;
  char* d_arena = nullptr;
  size_t arena_bytes = 0;
  // The stash: copies of the q of every refined patch, taken by
  // bsam_gpu_stash (old grids as TransferValues reads them), with records
  // whose q pointers point into it.
  char* d_stash = nullptr;
  size_t stash_cap = 0;
  // The hierarchy's tables (records, work lists, patch lists, overlap copies,
  // copy spans, tensor maps, partial sums) in one device buffer, grown and
  // never shrunk, filled by one copy from a host image per set_hierarchy.
  char* d_meta = nullptr;
  size_t meta_cap = 0;
  std::vector<unsigned char> meta_host;
  // The arena a regrid released, kept for the next hierarchy of no larger
  // size (regridding every step alternates between two arenas).
  char* spare_arena = nullptr;
  size_t spare_bytes = 0;
  bool regridding = false;  // set_hierarchy called by bsam_gpu_regrid
  // Task lists of bsam_gpu_regrid and bsam_gpu_errflags_level (grown, never
  // shrunk; both synchronise before returning, so one buffer serves both).
  char* d_regrid = nullptr;
  size_t regrid_cap = 0;
  std::vector<unsigned char> regrid_host;
  // Page-locked bounce buffer (grown, never shrunk) for the handle's copies
  // from and to pageable host memory; every user synchronises the stream
  // before the buffer is written again.
  void* h_pin = nullptr;
  size_t pin_cap = 0;
  bool attrs_set = false;      // the fused kernels' shared-memory attributes
  uint8_t* d_flags = nullptr;  // bsam_gpu_errflags_level's device flags
  int32_t* d_sat = nullptr;    // bsam_gpu_tag_level's summed-area tables
  size_t sat_cap = 0;
  CopySpan* d_qold_spans = nullptr;  // CopyQToQold: q -> qold of every patch that has qold
  int nqold_spans = 0;
  int64_t qold_span_max = 0;
  CopySpan* d_stash_spans = nullptr;
  size_t stash_spans_cap = 0;
  size_t flags_cap = 0;
  std::vector<DevPatch> stash_hp;
  std::vector<bsam_patch_desc> stash_desc;
  std::vector<LevelPlan> levels;     // index level - minlevel
  std::vector<int> masters;          // finest-level state patches
  Item* d_master = nullptr;          // tiles over the masters
  Item* d_state = nullptr;           // tiles over every state patch on levels >= 0
  int nstate = 0;
  Item* d_root = nullptr;            // tiles over the root patch (mass)
  int nroot = 0;
  bool amr = false;                  // levels above the root exist
  int* d_plist = nullptr;            // patch lists of the refined levels
  OverlapCopy* d_ovl = nullptr;      // their GhostOverlap transfers
  // Host copies of the refined levels' patch lists and transfers grouped by
  // destination, with per level the span of each (engine_view).
  std::vector<int> h_plist;
  std::vector<OverlapCopy> h_ovl_by_dst;
  std::vector<int2> h_ovl_range;
  std::vector<std::pair<int, int>> h_span_plist, h_span_ovl;
  int nmaster = 0;
  Item* d_items = nullptr;
  CUtensorMap* d_tmaps = nullptr;    // TMA maps of the fused levels' fields
  double* d_partials = nullptr;
  int max_items = 0;
  int* d_err = nullptr;  // kernel error flag (bounded waits that gave up)
  // Fused stages off by default: at L2-resident sizes the per-pass kernels
  // are faster; tests and tuning switch them on.
  bsam_tuning tuning{0, 64, 0, 0, 0, {0, 0, 0}};
  int bottom_level = -1000;  // levels <= this run inside k_bottom
  int* d_tops = nullptr;     // top patch of each k_bottom chain
  int ntops = 0;
  double denom = 1.0;        // nrvars * cells of the finest level (ErrorAFAS)
  cudaGraphExec_t step_exec = nullptr;  // V-cycle loop graph (built lazily)
  int graph_kernels_per_vcycle = 0;
  double* d_trace = nullptr;  // per-V-cycle residuals of the graph path
  double* h_trace = nullptr;  // pinned
  DevStatus* d_status = nullptr;
  DevStatus* h_status = nullptr;  // pinned
  std::vector<double> trace;
  std::string err;
  // instrumentation
  bool profiling = false;
  bsam_gpu_stats stats{};
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pool;
  size_t ev_used = 0;
  int64_t ev_cells = 0;   // cells of the finest V-cycle level
  int ev_bytes = 8;       // bytes per value on that level
};

namespace {

int fail(bsam_gpu* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

#define CU(call)                                                                  \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess)                                                        \
      return fail(h, BSAM_ERR_CUDA, std::string(__func__) + ":" + std::to_string(__LINE__) + \
                                        ": " #call ": " + cudaGetErrorString(e_));         \
  } while (0)

int64_t roundup(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

LevelPlan& plan(bsam_gpu* h, int level) { return h->levels[level - h->minlevel]; }

// The bounce buffer with room for `bytes`.  Copies through it are DMA
// copies queued on the stream; copies from pageable memory instead pass
// through the driver's staging, which handles regridding side by side on
// several host threads contend for.
void* pin_reserve(bsam_gpu* h, size_t bytes) {
  if (bytes > h->pin_cap) {
    if (h->h_pin) cudaFreeHost(h->h_pin);
    h->h_pin = nullptr;
    h->pin_cap = 0;
    const size_t want = std::max<size_t>(bytes + bytes / 2, (size_t)1 << 16);
    if (cudaMallocHost(&h->h_pin, want) != cudaSuccess) return nullptr;
    h->pin_cap = want;
  }
  return h->h_pin;
}

// Queues a host -> device copy of pageable `src` through the bounce buffer
// (the caller synchronises the stream before the buffer's next use).
int h2d_bounce(bsam_gpu* h, void* dst, const void* src, size_t bytes) {
  if (!bytes) return BSAM_OK;
  void* p = pin_reserve(h, bytes);
  if (!p) return fail(h, BSAM_ERR_NOMEM, "page-locked staging allocation failed");
  std::memcpy(p, src, bytes);
  CU(cudaMemcpyAsync(dst, p, bytes, cudaMemcpyHostToDevice, h->stream));
  return BSAM_OK;
}

// Device -> pageable host through the bounce buffer; waits for the stream.
int d2h_bounce(bsam_gpu* h, void* dst, const void* src, size_t bytes) {
  if (!bytes) return BSAM_OK;
  void* p = pin_reserve(h, bytes);
  if (!p) return fail(h, BSAM_ERR_NOMEM, "page-locked staging allocation failed");
  CU(cudaMemcpyAsync(p, src, bytes, cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  std::memcpy(dst, p, bytes);
  return BSAM_OK;
}

void tiles_for(int patch, const int* n, int ndims, std::vector<Item>& out) {
  const int tx = (n[0] + TILE_X - 1) / TILE_X;
  const int ty = (n[1] + TILE_Y - 1) / TILE_Y;
  const int tz = ndims == 3 ? n[2] : 1;
  for (int z = 0; z < tz; ++z)
    for (int y = 0; y < ty; ++y)
      for (int x = 0; x < tx; ++x) out.push_back(Item{patch, x, y, z});
}

dim3 block_dim() { return dim3(32, TILE_Y, 1); }

int elem_bytes(int prec) { return prec == PREC_F32 ? 4 : 8; }

// Timed finest-level smoothing stages: events are pooled and read back at
// the next host synchronisation (drain_events).
void stage_begin(bsam_gpu* h, int level) {
  if (!h->profiling || level != h->finestlevel) return;
  if (h->ev_used == h->ev_pool.size()) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    h->ev_pool.push_back({a, b});
  }
  cudaEventRecord(h->ev_pool[h->ev_used].first, h->stream);
}

void stage_end(bsam_gpu* h, int level) {
  if (!h->profiling || level != h->finestlevel) return;
  cudaEventRecord(h->ev_pool[h->ev_used].second, h->stream);
  ++h->ev_used;
}

void drain_events(bsam_gpu* h) {
  for (size_t e = 0; e < h->ev_used; ++e) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, h->ev_pool[e].first, h->ev_pool[e].second) == cudaSuccess) {
      h->stats.smooth_ms += ms;
      h->stats.smooth_stages += 1;
      h->stats.smooth_cells += h->ev_cells;
      h->stats.smooth_bytes += 6.0 * h->ev_bytes * (double)h->ev_cells;
    }
  }
  h->ev_used = 0;
}

// ---- typed launches -----------------------------------------------------------

template <class T, int D>
void launch_relax_t(bsam_gpu* h, const LevelPlan& L, int color) {
  k_relax<T, D><<<L.nfine, block_dim(), 0, h->stream>>>(h->d_patches, L.d_fine, color);
}

// what: 0 = RestrictSolution, 2 = CoarseLoadingFunction, 1 = CorrectFine.
template <class TC, class TP, int D>
void launch_transfer_t(bsam_gpu* h, const LevelPlan& L, int what) {
  if (what == 0)
    k_restrict<TC, TP, D><<<L.ncoarse, block_dim(), 0, h->stream>>>(h->d_patches, L.d_coarse);
  else if (what == 2)
    k_coarse_load<TC, TP, D><<<L.ncoarse, block_dim(), 0, h->stream>>>(h->d_patches, L.d_coarse);
  else
    k_correct<TC, TP, D><<<L.nfine, block_dim(), 0, h->stream>>>(h->d_patches, L.d_fine);
}

// SetGhost(level, ipass) of a refined level (boundary.f90:58-89): coarse-fine
// interpolation, sibling exchange, physical faces -- one launch (a CTA per
// patch runs the three in order).
// Levels at and below the root keep their ghosts by write-through.
void amr_ghost(bsam_gpu* h, int level, int ipass) {
  if (level < h->minlevel || level > h->finestlevel) return;
  const LevelPlan& L = plan(h, level);
  if (!L.amr) return;
  if (h->rp.ndims == 2) {
    k_ghost2<<<L.nplist, 128, 0, h->stream>>>(h->d_patches, L.d_plist, L.d_ovl_by_dst,
                                              L.d_ovl_range, ipass);
  } else {
    k_ghost3<<<L.nplist, 256, 0, h->stream>>>(h->d_patches, L.d_plist, L.d_ovl_by_dst,
                                              L.d_ovl_range, ipass);
  }
  ++h->stats.launches;
}

// GetCoarseGhostPoints for the children of a partly covered level: the
// snapshot qs of every parent patch becomes a full copy of q (taken after
// restriction and SetGhost).
void snapshot(bsam_gpu* h, int level) {
  const LevelPlan& L = plan(h, level);
  if (!L.snap) return;
  for (int p : L.patches) {
    const DevPatch& P = h->hp[p];
    if (!P.qs[0]) continue;  // not a parent: no child reads a snapshot of it
    const int64_t lead = 128 / sizeof(double) - 1;
    for (int c = 0; c < 2; ++c)
      cudaMemcpyAsync(static_cast<double*>(P.qs[c]) - lead, static_cast<double*>(P.q[c]) - lead,
                      h->field_elems[p] * sizeof(double), cudaMemcpyDeviceToDevice, h->stream);
  }
}

// FillDown(solutionfield) over the refined levels (afas:223-239): each
// level's q restricted into its parent, then the parent level's SetGhost.
// Below the root the same restriction is overwritten by RestrictSolution
// before any read, so it is not issued.
void filldown(bsam_gpu* h) {
  for (int level = h->finestlevel; level >= 1; --level) {
    const LevelPlan& L = plan(h, level);
    if (h->rp.ndims == 2)
      k_filldown<2><<<L.ncoarse, block_dim(), 0, h->stream>>>(h->d_patches, L.d_coarse);
    else
      k_filldown<3><<<L.ncoarse, block_dim(), 0, h->stream>>>(h->d_patches, L.d_coarse);
    ++h->stats.launches;
    amr_ghost(h, level - 1, 0);
  }
}

template <int D>
void launch_transfer_d(bsam_gpu* h, const LevelPlan& L, int pc, int pp, int what) {
  if (pc == PREC_F32 && pp == PREC_F32) launch_transfer_t<float, float, D>(h, L, what);
  else if (pc == PREC_F32) launch_transfer_t<float, double, D>(h, L, what);
  else launch_transfer_t<double, double, D>(h, L, what);
}

// LevelRelax (afas:523-547).  dir selects the buffers of a fused level:
// 0 = pre-smoothing (q -> qb), 1 = post-smoothing (qb -> q).
void relax_level(bsam_gpu* h, int level, int dir) {
  const LevelPlan& L = plan(h, level);
  stage_begin(h, level);
  if (L.fused) {
    if (L.prec == PREC_F32)
      k_smooth3_fused<float><<<L.nfused, Fused3<float>::THREADS, Fused3<float>::SMEM, h->stream>>>(
          h->d_patches, L.d_fused, dir, 0, h->d_err);
    else
      k_smooth3_fused<double><<<L.nfused, Fused3<double>::THREADS, Fused3<double>::SMEM,
                                h->stream>>>(h->d_patches, L.d_fused, dir, 0, h->d_err);
    ++h->stats.launches;
  } else {
    for (int pass = 0; pass < h->rp.nsmoothingpasses; ++pass)
      for (int color = 0; color < 2; ++color) {
        if (h->rp.ndims == 2) {
          if (L.prec == PREC_F32) launch_relax_t<float, 2>(h, L, color);
          else launch_relax_t<double, 2>(h, L, color);
        } else {
          if (L.prec == PREC_F32) launch_relax_t<float, 3>(h, L, color);
          else launch_relax_t<double, 3>(h, L, color);
        }
        ++h->stats.launches;
        amr_ghost(h, level, color + 1);  // SetGhost(level, ipass) (afas:542)
      }
  }
  stage_end(h, level);
}

// what 0: RestrictSolution, parent SetGhost(level-1, 0), GetCoarseGhostPoints
// and CoarseLoadingFunction (afas:503-509); what 1: CorrectFine and
// SetGhost(level, 0) (afas:513-515).
void transfer(bsam_gpu* h, int level, int what) {
  const LevelPlan& L = plan(h, level);
  const int pp = plan(h, level - 1).prec;
  auto launch = [&](int w) {
    if (h->rp.ndims == 2) launch_transfer_d<2>(h, L, L.prec, pp, w);
    else launch_transfer_d<3>(h, L, L.prec, pp, w);
    ++h->stats.launches;
  };
  if (what == 0) {
    launch(0);
    amr_ghost(h, level - 1, 0);
    snapshot(h, level - 1);
    launch(2);
  } else {
    launch(1);
    amr_ghost(h, level, 0);
  }
}

// AFASVcycle (afas:488-521).
void vcycle(bsam_gpu* h, int level) {
  if (level == h->bottom_level) {
    // AFASVcycle(level) down to the coarsest level in one launch (bottom.cuh);
    // bottom levels are FP64 in both forms.
    if (h->rp.ndims == 2)
      k_bottom<double, 2><<<h->ntops, BOTTOM_THREADS, 0, h->stream>>>(h->d_patches, h->d_tops,
                                                                      h->rp.nsmoothingpasses);
    else
      k_bottom<double, 3><<<h->ntops, BOTTOM_THREADS, 0, h->stream>>>(h->d_patches, h->d_tops,
                                                                      h->rp.nsmoothingpasses);
    ++h->stats.launches;
    return;
  }
  relax_level(h, level, 0);  // LevelRelax (afas:499)
  if (level > h->minlevel) {
    transfer(h, level, 0);   // RestrictSolution + CoarseLoadingFunction (afas:503-509)
    vcycle(h, level - 1);    // afas:511
    transfer(h, level, 1);   // CorrectFine (afas:513)
    relax_level(h, level, 1);  // afas:517
  }
}

// ErrorAFAS on the finest level (afas:94, 108-221) into d_status.  In the
// mixed form the same FP64 norm is taken by k_defect, which also prepares
// the twins for the next FP32 V-cycle.
void launch_resid(bsam_gpu* h) {
  const int nd = h->rp.ndims;
  const dim3 b = block_dim();
  if (!h->mixed) {
    if (nd == 2)
      k_resid_norm<double, 2><<<h->nmaster, b, 0, h->stream>>>(
          h->d_patches, h->d_master, h->d_partials, h->d_status, h->nmaster, h->denom,
          h->rp.qerrortol);
    else
      k_resid_norm<double, 3><<<h->nmaster, b, 0, h->stream>>>(
          h->d_patches, h->d_master, h->d_partials, h->d_status, h->nmaster, h->denom,
          h->rp.qerrortol);
  } else {
    const bool f32 = plan(h, h->finestlevel).prec == PREC_F32;
#define DEFECT(TW, D)                                                                        \
  k_defect<TW, D><<<h->nmaster, b, 0, h->stream>>>(h->d_patches, h->d_master, h->d_partials, \
                                                   h->d_status, h->nmaster, h->denom,        \
                                                   h->rp.qerrortol)
    if (nd == 2) {
      if (f32) DEFECT(float, 2);
      else DEFECT(double, 2);
    } else {
      if (f32) DEFECT(float, 3);
      else DEFECT(double, 3);
    }
#undef DEFECT
  }
  ++h->stats.launches;
}

// Mixed form: q64 += q32 - fl32(q64) after the FP32 V-cycle.
void launch_update(bsam_gpu* h) {
  const int nd = h->rp.ndims;
  const bool f32 = plan(h, h->finestlevel).prec == PREC_F32;
  const dim3 b = block_dim();
  if (nd == 2) {
    if (f32) k_update<float, 2><<<h->nmaster, b, 0, h->stream>>>(h->d_patches, h->d_master);
    else k_update<double, 2><<<h->nmaster, b, 0, h->stream>>>(h->d_patches, h->d_master);
  } else {
    if (f32) k_update<float, 3><<<h->nmaster, b, 0, h->stream>>>(h->d_patches, h->d_master);
    else k_update<double, 3><<<h->nmaster, b, 0, h->stream>>>(h->d_patches, h->d_master);
  }
  ++h->stats.launches;
}

// One outer iteration of MultigridIterations: V-cycle, then ErrorAFAS.
void iteration(bsam_gpu* h) {
  vcycle(h, h->finestlevel);
  if (h->mixed) launch_update(h);
  if (h->amr) filldown(h);  // FillDown(solutionfield) after the V-cycle (afas:73)
  launch_resid(h);
}

// Captures the V-cycle loop of MultigridIterations (afas:69-104) as a graph
// with one conditional WHILE node whose body is one iteration + k_mg_loop;
// k_mg_loop sets the condition.  The default value 1 makes the body run at
// least once per launch, as the reference's loop does.
int build_step_graph(bsam_gpu* h) {
  cudaGraph_t g = nullptr;
  CU(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle handle;
  cudaError_t e = cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault);
  cudaGraphNodeParams np{};
  cudaGraphNode_t node;
  if (e == cudaSuccess) {
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = handle;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    e = cudaGraphAddNode(&node, g, nullptr, 0, &np);
  }
  if (e == cudaSuccess) {
    cudaGraph_t body = np.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(h->stream, body, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      const int64_t before = h->stats.launches;
      iteration(h);
      k_mg_loop<<<1, 1, 0, h->stream>>>(h->d_status, h->d_trace, h->rp.maxvcycles,
                                         h->rp.qerrortol, handle);
      h->graph_kernels_per_vcycle = (int)(h->stats.launches - before) + 1;
      h->stats.launches = before;
      cudaGraph_t captured = nullptr;
      e = cudaStreamEndCapture(h->stream, &captured);
    }
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&h->step_exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    h->step_exec = nullptr;
    cudaGetLastError();
    return fail(h, BSAM_ERR_CUDA, std::string("step graph: ") + cudaGetErrorString(e));
  }
  return BSAM_OK;
}

// SetBC on the FP64 state patches of one level.
int ghost_level(bsam_gpu* h, int level) {
  for (int p = 0; p < h->nuser; ++p) {
    const DevPatch& P = h->hp[p];
    if (P.level != level || P.prec != PREC_F64 || P.delta) continue;
    int64_t total = (int64_t)(P.n[0] + 2) * (P.n[1] + 2) * (h->rp.ndims == 3 ? P.n[2] + 2 : 1);
    int nb = (int)((total + 255) / 256);
    if (h->rp.ndims == 2) k_setbc<double, 2><<<nb, 256, 0, h->stream>>>(h->d_patches, p, total);
    else k_setbc<double, 3><<<nb, 256, 0, h->stream>>>(h->d_patches, p, total);
    ++h->stats.launches;
  }
  return BSAM_OK;
}

int face_rule(int ndims, int face, int code, int* rule) {
  if (code == 1) {
    *rule = BC_COPY;
  } else if (code >= 10 && code <= 99) {
    // UserBC2D: faces 1,2 -> 2 - q (all vars); faces 3,4 -> copy of vars 1,2.
    // UserBC3D: every face -> 2 - q (problem.f90:646-756).
    *rule = (ndims == 2 && face >= 2) ? BC_COPY : BC_REFLECT;
  } else if (code == 999) {
    *rule = BC_NONE;
  } else if (code == 2) {
    *rule = BC_PERIODIC;  // both faces of the dimension (checked by the caller)
  } else {
    return -1;
  }
  return 0;
}

int64_t cells_of(const int* mx, int nd) {
  int64_t c = 1;
  for (int n = 0; n < nd; ++n) c *= mx[n];
  return c;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// 3D map of one field of patch P: the array from its allocation start
// (`lead` elements before element (0,0,0)), dims (sy, n1+2, n2+2), box
// (hx, hy, 1).  Returns false if the driver rejects it.
bool encode_field_map(CUtensorMap* m, const DevPatch& P, const void* field, int hx, int hy) {
  auto enc = tensor_map_encoder();
  if (!enc) return false;
  const int es = elem_bytes(P.prec);
  const int64_t lead = 128 / es - 1;
  void* base = (char*)field - lead * es;
  const cuuint64_t dims[3] = {(cuuint64_t)P.sy, (cuuint64_t)(P.n[1] + 2),
                              (cuuint64_t)(P.n[2] + 2)};
  const cuuint64_t strides[2] = {(cuuint64_t)(P.sy * es), (cuuint64_t)(P.sz * es)};
  const cuuint32_t box[3] = {(cuuint32_t)hx, (cuuint32_t)hy, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r =
      enc(m, P.prec == PREC_F32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
          3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace

namespace bsam {

int engine_view(bsam_gpu* h, EngineView& v) {
  if (!h || !h->have_hierarchy) return BSAM_ERR_STATE;
  v.ndims = h->rp.ndims;
  v.minlevel = h->minlevel;
  v.finestlevel = h->finestlevel;
  v.nsmoothingpasses = h->rp.nsmoothingpasses;
  v.maxvcycles = h->rp.maxvcycles;
  v.mixed = h->mixed;
  v.qerrortol = h->rp.qerrortol;
  v.denom = h->denom;
  v.recs = h->hp;
  v.masters = h->masters;
  v.levels.assign(h->levels.size(), EngineLevelView{});
  for (size_t li = 0; li < h->levels.size(); ++li) {
    const LevelPlan& L = h->levels[li];
    EngineLevelView& E = v.levels[li];
    E.level = L.level;
    E.amr = L.amr;
    E.snap = L.snap;
    E.patches = L.patches;
    if (!L.amr || li >= h->h_span_plist.size()) continue;
    const auto sp = h->h_span_plist[li], so = h->h_span_ovl[li];
    E.ovl.assign(h->h_ovl_by_dst.begin() + so.first,
                 h->h_ovl_by_dst.begin() + so.first + so.second);
    E.range.assign(h->h_ovl_range.begin() + sp.first,
                   h->h_ovl_range.begin() + sp.first + sp.second);
  }
  return BSAM_OK;
}

int engine_prologue(bsam_gpu* h) {
  if (!h || !h->have_hierarchy) return BSAM_ERR_STATE;
  if (h->mixed) return fail(h, BSAM_ERR_UNSUPPORTED, "the batch runs refined hierarchies in FP64");
  CU(cudaSetDevice(h->device));
  if (h->amr) filldown(h);
  if (h->rp.ndims == 2)
    k_source<double, 2><<<h->nstate, block_dim(), 0, h->stream>>>(h->d_patches, h->d_state);
  else
    k_source<double, 3><<<h->nstate, block_dim(), 0, h->stream>>>(h->d_patches, h->d_state);
  ++h->stats.launches;
  CU(cudaGetLastError());
  return BSAM_OK;
}

cudaStream_t engine_stream(bsam_gpu* h) { return h ? h->stream : nullptr; }

int engine_device(bsam_gpu* h) { return h ? h->device : -1; }

}  // namespace bsam

extern "C" {

const char* bsam_gpu_strerror(int code) {
  switch (code) {
    case BSAM_OK: return "ok";
    case BSAM_ERR_ARG: return "invalid argument";
    case BSAM_ERR_CUDA: return "CUDA runtime error";
    case BSAM_ERR_NOMEM: return "device memory allocation failed";
    case BSAM_ERR_STATE: return "call out of order";
    case BSAM_ERR_UNSUPPORTED: return "configuration not supported";
    case BSAM_ERR_NODEVICE: return "no usable CUDA device";
    case BSAM_ERR_DIVERGED: return "non-finite residual";
    case BSAM_ERR_TOO_LARGE: return "patch exceeds the static scratch limit of the no-alloc entry point";
    default: return "unknown status";
  }
}

const char* bsam_gpu_last_error(bsam_gpu* h) { return h ? h->err.c_str() : "null handle"; }

int bsam_gpu_create(bsam_gpu** out, int device, const bsam_run_params* p) {
  bsam_gpu* h = nullptr;
  if (!out || !p) return BSAM_ERR_ARG;
  *out = nullptr;
  if (p->ndims < 2 || p->ndims > 3 || p->nrvars != 2 || p->mbc != 1 || p->maux != 0 ||
      p->errortype != 1 || p->nsmoothingpasses < 1 || p->maxvcycles < 1)
    return BSAM_ERR_UNSUPPORTED;
  if (p->precision != BSAM_PREC_FP64 && p->precision != BSAM_PREC_MIXED)
    return BSAM_ERR_UNSUPPORTED;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0)
    return BSAM_ERR_NODEVICE;
  h = new bsam_gpu();
  h->device = device;
  h->rp = *p;
  h->mixed = p->precision == BSAM_PREC_MIXED;
  if (cudaSetDevice(device) != cudaSuccess) {
    delete h;
    return BSAM_ERR_NODEVICE;
  }
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&h->d_status, sizeof(DevStatus)) != cudaSuccess ||
      cudaMallocHost(&h->h_status, sizeof(DevStatus)) != cudaSuccess) {
    delete h;
    return BSAM_ERR_CUDA;
  }
  cudaMemset(h->d_status, 0, sizeof(DevStatus));
  h->d_err = &h->d_status->kerr;
  *out = h;
  return BSAM_OK;
}

static void free_hierarchy(bsam_gpu* h) {
  // d_items, d_tmaps, d_tops, d_patches, d_partials, d_qold_spans, d_plist
  // and d_ovl point into d_meta, which the handle keeps.
  h->d_tmaps = nullptr;
  if (h->step_exec) cudaGraphExecDestroy(h->step_exec);
  if (h->d_arena) cudaFree(h->d_arena);
  h->d_qold_spans = nullptr;
  h->nqold_spans = 0;
  h->qold_span_max = 0;
  h->d_items = nullptr;
  h->d_tops = nullptr;
  h->ntops = 0;
  h->step_exec = nullptr;
  h->d_arena = nullptr;
  h->d_patches = nullptr;
  h->d_partials = nullptr;
  h->d_master = nullptr;
  h->nmaster = 0;
  h->d_state = h->d_root = nullptr;
  h->nstate = h->nroot = 0;
  h->d_plist = nullptr;
  h->d_ovl = nullptr;
  h->amr = false;
  h->levels.clear();
  h->masters.clear();
  h->hp.clear();
  h->desc.clear();
  h->field_elems.clear();
  h->have_hierarchy = false;
}

int bsam_gpu_set_hierarchy(bsam_gpu* h, int npatch, const bsam_patch_desc* patches,
                           int finestlevel) {
  if (!h || npatch <= 0 || !patches) return BSAM_ERR_ARG;
  CU(cudaSetDevice(h->device));
  free_hierarchy(h);
  const int nd = h->rp.ndims;
  int minlevel = patches[0].level;
  for (int p = 0; p < npatch; ++p) minlevel = std::min(minlevel, patches[p].level);
  if (finestlevel < 0 || minlevel > 0) return fail(h, BSAM_ERR_ARG, "levels out of range");
  if (finestlevel > 0 && h->mixed)
    return fail(h, BSAM_ERR_UNSUPPORTED,
                "levels above the root are built for the FP64 form (no mixed-precision AMR)");
  h->amr = finestlevel > 0;
  h->minlevel = minlevel;
  h->finestlevel = finestlevel;
  h->nuser = npatch;
  h->levels.assign(finestlevel - minlevel + 1, LevelPlan{});
  for (int l = minlevel; l <= finestlevel; ++l) plan(h, l).level = l;
  h->desc.assign(patches, patches + npatch);

  // Bottom level: the finest level such that it and every coarser level hold
  // at most bottom_cells cells per patch (uniform hierarchies only).
  h->bottom_level = -1000;
  // Default: chains from 1024 cells (2D) or 512 (3D) down.  The one-CTA
  // chain runs on a single SM, so a larger top level there (4096 cells: 64^2,
  // 16^3) leaves the rest of the GPU idle for longer than the grid kernels
  // take for it (measured: 128^2 FP64 829 -> 915 time-steps/s; 16^3 .. 1^3
  // alone was a quarter of a 128^3 V-cycle).
  const bool dflt = h->tuning.bottom_cells == 0;
  const int bmax = dflt ? (nd == 3 ? DEFAULT_BOTTOM_CELLS_3D : DEFAULT_BOTTOM_CELLS_2D)
                        : h->tuning.bottom_cells;
  if (bmax > 0) {
    // Only the root and the levels below it (one uniform patch each).
    for (int l = minlevel; l <= std::min(finestlevel, 0); ++l) {
      bool small = true;
      for (int p = 0; p < npatch; ++p)
        if (patches[p].level == l) small = small && cells_of(patches[p].mx, nd) <= bmax;
      if (!small) break;
      h->bottom_level = l;
    }
    if (h->bottom_level - minlevel + 1 > BOTTOM_MAX_DEPTH) h->bottom_level = -1000;
  }
  // Mixed form: levels at or below this size stay FP64 -- the levels the
  // bottom kernel runs, including the coarsest; 4096 cells under the default
  // bottom size and when the bottom kernel is switched off (the levels
  // between the default bottom and 4096 cells run FP64 grid kernels, which
  // give the bottom kernel's bits).
  const int64_t fp64_cells = (!dflt && bmax > 0) ? (int64_t)bmax : MIXED_FP64_CELLS;

  // Records: the caller's patches, then one twin per finest-level patch in
  // the mixed form.
  std::vector<int> twin_of(npatch, -1);
  int nrec = npatch;
  for (int p = 0; p < npatch; ++p)
    if (patches[p].level == finestlevel) {
      h->masters.push_back(p);
      if (h->mixed) twin_of[p] = nrec++;
    }
  h->hp.assign(nrec, DevPatch{});
  h->field_elems.assign(nrec, 0);
  // rec_src[r]: the caller's patch whose geometry record r has.
  std::vector<int> rec_src(nrec);
  for (int p = 0; p < npatch; ++p) {
    rec_src[p] = p;
    if (twin_of[p] >= 0) rec_src[twin_of[p]] = p;
  }

  const double eps2 = h->rp.eps * h->rp.eps;
  size_t total = 0;
  std::vector<size_t> offs(nrec);
  std::vector<int> nfields(nrec, 0);
  std::vector<char> want_qold(nrec, 0), want_qs(nrec, 0);
  for (int r = 0; r < nrec; ++r) {
    const int p = rec_src[r];
    const bool is_twin = r >= npatch;
    const bsam_patch_desc& d = patches[p];
    if (d.level < minlevel || d.level > finestlevel)
      return fail(h, BSAM_ERR_ARG, "patch level out of range");
    DevPatch& P = h->hp[r];
    P.ndims = nd;
    for (int n = 0; n < 3; ++n) {
      P.n[n] = n < nd ? d.mx[n] : 1;
      if (P.n[n] <= 0) return fail(h, BSAM_ERR_ARG, "mx must be positive");
    }
    P.parent = d.parent;
    P.level = d.level;
    P.problem = 0;
    P.active = 1;
    P.newstep = 0;
    P.twin = is_twin ? -1 : twin_of[p];
    P.master = is_twin ? p : -1;
    // Precision of the record.
    const int64_t ncell = cells_of(P.n, nd);
    if (!h->mixed || (!is_twin && d.level == finestlevel) || ncell <= fp64_cells)
      P.prec = PREC_F64;
    else
      P.prec = PREC_F32;
    if (d.parent >= 0) {
      if (d.parent >= npatch || patches[d.parent].level != d.level - 1)
        return fail(h, BSAM_ERR_ARG, "parent must be a patch on the next coarser level");
      for (int n = 0; n < nd; ++n) {
        if (P.n[n] % 2) return fail(h, BSAM_ERR_ARG, "a patch with a parent needs even mx");
        P.cn[n] = P.n[n] / 2;
        P.off[n] = d.mbounds[n][0] - 1;
        if (d.mbounds[n][1] - d.mbounds[n][0] + 1 != P.cn[n] || P.off[n] < 0 ||
            d.mbounds[n][1] > patches[d.parent].mx[n])
          return fail(h, BSAM_ERR_ARG, "mbounds inconsistent with mx / parent");
      }
    } else if (d.level != minlevel) {
      return fail(h, BSAM_ERR_ARG, "only the coarsest level may lack a parent");
    }
    for (int n = nd; n < 3; ++n) {
      P.cn[n] = 1;
      P.off[n] = 0;
    }
    P.wt = 1;
    for (int f = 0; f < 6; ++f) {
      if (f >= 2 * nd) {
        P.bc[f] = BC_NONE;
        continue;
      }
      int rule;
      if (face_rule(nd, f, d.mthbc[f], &rule))
        return fail(h, BSAM_ERR_UNSUPPORTED, "boundary code not supported");
      P.bc[f] = rule;
      P.code[f] = d.mthbc[f];
      if (rule == BC_NONE) P.wt = 0;
    }
    if (!P.wt && d.level < 1)
      return fail(h, BSAM_ERR_UNSUPPORTED, "internal faces occur only on refined levels");
    // Periodic faces (PeriodicSetup, boundary.f90:893-963): in pairs (the
    // reference stops otherwise, bsamroutines.f90:307-316), on hierarchies
    // without refined levels (TransferPeriodicBC between refined grids has no
    // device form here), and on dimensions whose extent is even or 1: with an
    // odd extent above 1 the first and last cells of the dimension have the
    // same colour, and a colour pass would read the periodic ghost that its
    // opposite cell writes through in the same pass.
    for (int n = 0; n < nd; ++n) {
      const bool lo = P.bc[2 * n] == BC_PERIODIC, hi = P.bc[2 * n + 1] == BC_PERIODIC;
      if (lo != hi) return fail(h, BSAM_ERR_ARG, "periodic faces come in pairs");
      if (lo && finestlevel > 0)
        return fail(h, BSAM_ERR_UNSUPPORTED, "periodic faces with refined levels");
      if (lo && P.n[n] > 1 && P.n[n] % 2)
        return fail(h, BSAM_ERR_UNSUPPORTED, "periodic dimension with an odd extent above 1");
    }
    // Does the V-cycle run on this record?  (Not on the masters of the mixed form.)
    const bool in_vcycle = !(h->mixed && !is_twin && d.level == finestlevel);
    // Mixed form: the V-cycle levels carry a correction of the master state
    // (mixed.cuh); a reflecting face maps a correction to its negative.
    P.delta = (h->mixed && in_vcycle) ? 1 : 0;
    if (P.delta)
      for (int f = 0; f < 2 * nd; ++f)
        if (P.bc[f] == BC_REFLECT) P.bc[f] = BC_NEGATE;
    // Fused stages: 3D V-cycle levels with a parent above the bottom, all
    // faces physical (the stage derives face ghosts from the tile itself).
    const int fmin = std::max(8, h->tuning.fuse_min_n);
    bool periodic = false;
    for (int f = 0; f < 2 * nd; ++f) periodic |= P.bc[f] == BC_PERIODIC;
    P.fused = (h->tuning.fuse_smoother != 0 && nd == 3 && finestlevel == 0 && in_vcycle &&
               d.parent >= 0 && !periodic &&
               d.level > h->bottom_level && !(P.delta && P.prec == PREC_F64) &&
               P.n[0] >= fmin && P.n[1] >= fmin && P.n[2] >= fmin)
                  ? 1
                  : 0;
    if (P.fused) {
      const int ftx = P.prec == PREC_F32 ? Fused3<float>::TX : Fused3<double>::TX;
      const int fty = P.prec == PREC_F32 ? Fused3<float>::TY : Fused3<double>::TY;
      const int tiles = ((P.n[0] + ftx - 1) / ftx) * ((P.n[1] + fty - 1) / fty);
      int chunk = h->tuning.chunk;
      if (chunk <= 0) {
        // About one CTA per SM, chunks of at least 16 planes.
        const int nchunk = std::max(1, std::min(148 / std::max(tiles, 1), P.n[2] / 16));
        chunk = (P.n[2] + nchunk - 1) / nchunk;
      }
      P.zchunk = std::max(1, std::min(chunk, P.n[2]));
    }
    // Layout: rows aligned to 128 bytes; the slack after the last row keeps
    // the fused kernel's halo'd row copies inside the allocation.
    const int es = elem_bytes(P.prec);
    const int64_t A = 128 / es, lead = A - 1;
    P.sy = roundup(lead + P.n[0] + 2, A);
    P.sz = nd == 3 ? P.sy * (P.n[1] + 2) : 0;
    const int64_t vol = nd == 3 ? P.sz * (P.n[2] + 2) : P.sy * (P.n[1] + 2);
    h->field_elems[r] = roundup(lead + vol + 64, 256 / es);
    offs[r] = total;
    bool parent_of_any = false;
    if (in_vcycle)
      for (int c = 0; c < npatch; ++c) parent_of_any |= patches[c].parent == p;
    const bool has_qold = !is_twin && d.level >= 0 && P.prec == PREC_F64 &&
                          (!h->mixed || d.level == finestlevel);
    nfields[r] = 2 /*q*/ + 2 /*f*/ + (has_qold ? 2 : 0) + (parent_of_any ? 2 : 0) +
                 (P.fused ? 2 : 0) + (P.delta ? 1 : 0);
    total += (size_t)h->field_elems[r] * nfields[r] * es;
    // Problem constants (problem.f90:183-187): h2 = h*h; dt/h2; eps2/h2; 2d*eps2/h2.
    P.h = d.dx;
    const double h2 = d.dx * d.dx;
    P.dt = h->rp.dt;
    P.eps2 = eps2;
    P.alpha = h->rp.alpha;
    P.tmp1 = h->rp.dt / h2;
    P.tmp2 = eps2 / h2;
    P.tmp3 = (2.0 * nd) * eps2 / h2;
    if (in_vcycle) plan(h, d.level).patches.push_back(r);
    want_qold[r] = has_qold;
    want_qs[r] = parent_of_any;
  }
  if (h->spare_arena && h->spare_bytes >= total) {
    h->d_arena = h->spare_arena;
    total = h->spare_bytes;
    h->spare_arena = nullptr;
    h->spare_bytes = 0;
  } else {
    // Under regridding the arena alternates with the spare: a quarter more
    // than this table needs lets the next tables of similar size reuse it.
    if (h->regridding) total += total / 4;
    if (cudaMalloc(&h->d_arena, total) != cudaSuccess)
      return fail(h, BSAM_ERR_NOMEM, "arena allocation failed");
  }
  h->arena_bytes = total;
  CU(cudaMemsetAsync(h->d_arena, 0, total, h->stream));
  for (int r = 0; r < nrec; ++r) {
    DevPatch& P = h->hp[r];
    const int es = elem_bytes(P.prec);
    char* base = h->d_arena + offs[r];
    const int64_t fe = h->field_elems[r], lead = 128 / es - 1;
    int slot = 0;
    auto next = [&]() { return (void*)(base + (fe * (slot++) + lead) * es); };
    const bool has_qold = want_qold[r], has_qs = want_qs[r];
    P.q[0] = next();
    P.q[1] = next();
    P.f[0] = next();
    P.f[1] = next();
    P.qo[0] = P.qo[1] = nullptr;
    P.qs[0] = P.qs[1] = nullptr;
    if (has_qold) {
      P.qo[0] = next();
      P.qo[1] = next();
    }
    if (has_qs) {
      P.qs[0] = next();
      P.qs[1] = next();
    }
    if (P.fused) {
      P.qb[0] = next();
      P.qb[1] = next();
    }
    P.bs = P.delta ? next() : nullptr;
  }
  // CopyQToQold as one launch: the whole field allocation of q onto qold's.
  std::vector<CopySpan> qold_spans;
  {
    std::vector<CopySpan>& spans = qold_spans;
    for (int r = 0; r < npatch; ++r) {
      const DevPatch& P = h->hp[r];
      if (!P.qo[0]) continue;
      const int64_t lead = 128 / sizeof(double) - 1;
      for (int c = 0; c < 2; ++c)
        spans.push_back(CopySpan{static_cast<const double*>(P.q[c]) - lead,
                                 static_cast<double*>(P.qo[c]) - lead, h->field_elems[r]});
      h->qold_span_max = std::max(h->qold_span_max, h->field_elems[r]);
    }
    h->nqold_spans = (int)spans.size();
  }
  // Parents of the twins are the masters' parents.
  for (int r = npatch; r < nrec; ++r) h->hp[r].parent = h->hp[rec_src[r]].parent;
  for (int r = 0; r < nrec; ++r)
    h->hp[r].pprec = h->hp[r].parent >= 0 ? h->hp[h->hp[r].parent].prec : h->hp[r].prec;
  // TMA tensor maps of the fused records (q0, q1, qb0, qb1, f0, f1, bs).
  std::vector<int> fused_recs;
  std::vector<CUtensorMap> maps;
  {
    for (int r = 0; r < nrec; ++r)
      if (h->hp[r].fused) fused_recs.push_back(r);
    if (!fused_recs.empty()) {
      maps.resize(7 * fused_recs.size());
      for (size_t k = 0; k < fused_recs.size(); ++k) {
        const DevPatch& P = h->hp[fused_recs[k]];
        const int hx = P.prec == PREC_F32 ? Fused3<float>::HX : Fused3<double>::HX;
        const int hy = P.prec == PREC_F32 ? Fused3<float>::HY : Fused3<double>::HY;
        const void* fields[7] = {P.q[0], P.q[1], P.qb[0], P.qb[1],
                                 P.f[0], P.f[1], P.bs ? P.bs : P.q[0]};
        for (int m = 0; m < 7; ++m)
          if (!encode_field_map(&maps[7 * k + m], P, fields[m], hx, hy))
            return fail(h, BSAM_ERR_CUDA, "cuTensorMapEncodeTiled rejected a field map");
      }

    }
  }

  // Level precisions and work lists.
  std::vector<Item> all;
  const size_t nl = h->levels.size();
  std::vector<std::pair<int, int>> spans_fine(nl), spans_coarse(nl), spans_fused(nl);
  for (size_t li = 0; li < nl; ++li) {
    LevelPlan& L = h->levels[li];
    if (L.patches.empty()) return fail(h, BSAM_ERR_ARG, "a level between minlevel and finest is empty");
    L.prec = h->hp[L.patches[0]].prec;
    for (int p : L.patches)
      if (h->hp[p].prec != L.prec) return fail(h, BSAM_ERR_ARG, "mixed precisions on one level");
    int s = (int)all.size();
    for (int p : L.patches) tiles_for(p, h->hp[p].n, nd, all);
    spans_fine[li] = {s, (int)all.size() - s};
    s = (int)all.size();
    for (int p : L.patches)
      if (h->hp[p].parent >= 0) tiles_for(p, h->hp[p].cn, nd, all);
    spans_coarse[li] = {s, (int)all.size() - s};
    // A level runs fused stages only when every patch on it does.
    L.fused = true;
    for (int p : L.patches) L.fused = L.fused && h->hp[p].fused;
    if (!L.fused)
      for (int p : L.patches) h->hp[p].fused = 0;
    s = (int)all.size();
    if (L.fused)
      for (int p : L.patches) {
        const DevPatch& P = h->hp[p];
        const int ftx = P.prec == PREC_F32 ? Fused3<float>::TX : Fused3<double>::TX;
        const int fty = P.prec == PREC_F32 ? Fused3<float>::TY : Fused3<double>::TY;
        const int tx = (P.n[0] + ftx - 1) / ftx;
        const int ty = (P.n[1] + fty - 1) / fty;
        const int tz = (P.n[2] + P.zchunk - 1) / P.zchunk;
        for (int z = 0; z < tz; ++z)
          for (int y = 0; y < ty; ++y)
            for (int x = 0; x < tx; ++x) all.push_back(Item{p, x, y, z});
      }
    spans_fused[li] = {s, (int)all.size() - s};
  }
  const int s_master = (int)all.size();
  for (int p : h->masters) tiles_for(p, h->hp[p].n, nd, all);
  h->nmaster = (int)all.size() - s_master;
  // State patches (levels >= root, the caller's records) and the root.
  const int s_state = (int)all.size();
  for (int p = 0; p < npatch; ++p)
    if (patches[p].level >= 0) tiles_for(p, h->hp[p].n, nd, all);
  h->nstate = (int)all.size() - s_state;
  const int s_root = (int)all.size();
  for (int p = 0; p < npatch; ++p)
    if (patches[p].level == 0) tiles_for(p, h->hp[p].n, nd, all);
  h->nroot = (int)all.size() - s_root;
  // Refined levels: patch lists and GhostOverlap transfers
  // (ApplyOnLevelPairs order: each patch with every later one).
  std::vector<int> plist_all;
  std::vector<OverlapCopy> ovl_all;
  std::vector<std::pair<int, int>> span_plist(nl), span_ovl(nl);
  for (size_t li = 0; li < nl; ++li) {
    LevelPlan& L = h->levels[li];
    L.amr = L.level >= 1;
    L.snap = L.level >= 0 && L.level < finestlevel;
    span_plist[li] = {(int)plist_all.size(), 0};
    span_ovl[li] = {(int)ovl_all.size(), 0};
    if (!L.amr) continue;
    for (int p : L.patches) plist_all.push_back(p);
    for (size_t a = 0; a < L.patches.size(); ++a)
      for (size_t bi = a + 1; bi < L.patches.size(); ++bi) {
        const bsam_patch_desc& g1 = patches[L.patches[a]];
        const bsam_patch_desc& g2 = patches[L.patches[bi]];
        int ov[3][2] = {{1, 1}, {1, 1}, {1, 1}};
        bool empty = false;
        for (int n = 0; n < nd; ++n) {
          ov[n][0] = std::max(g1.mglobal[n][0] - 1, g2.mglobal[n][0] - 1);
          ov[n][1] = std::min(g1.mglobal[n][1] + 1, g2.mglobal[n][1] + 1);
          empty |= ov[n][1] < ov[n][0];
        }
        if (empty) continue;
        // dst takes the other grid's interior inside the overlap.
        auto emit = [&](int dst, const bsam_patch_desc& gd, int src, const bsam_patch_desc& gs) {
          int box[3][2] = {{1, 1}, {1, 1}, {1, 1}};
          for (int n = 0; n < nd; ++n) {
            box[n][0] = std::max(ov[n][0], gs.mglobal[n][0]);
            box[n][1] = std::min(ov[n][1], gs.mglobal[n][1]);
            if (box[n][1] < box[n][0]) return;
          }
          OverlapCopy o;
          o.dst = dst;
          o.src = src;
          o.i0 = box[0][0] - gd.mglobal[0][0] + 1;
          o.i1 = box[0][1] - gd.mglobal[0][0] + 1;
          o.j0 = box[1][0] - gd.mglobal[1][0] + 1;
          o.j1 = box[1][1] - gd.mglobal[1][0] + 1;
          o.di = gd.mglobal[0][0] - gs.mglobal[0][0];
          o.dj = gd.mglobal[1][0] - gs.mglobal[1][0];
          if (nd == 3) {
            o.k0 = box[2][0] - gd.mglobal[2][0] + 1;
            o.k1 = box[2][1] - gd.mglobal[2][0] + 1;
            o.dk = gd.mglobal[2][0] - gs.mglobal[2][0];
          } else {
            o.k0 = o.k1 = 0;
            o.dk = 0;
          }
          ovl_all.push_back(o);
        };
        emit(L.patches[a], g1, L.patches[bi], g2);
        emit(L.patches[bi], g2, L.patches[a], g1);
      }
    span_plist[li].second = (int)plist_all.size() - span_plist[li].first;
    span_ovl[li].second = (int)ovl_all.size() - span_ovl[li].first;
  }
  // Per level: the overlap transfers grouped by destination (stable), with
  // each patch-list entry's {first, count} relative to the level's group.
  std::vector<OverlapCopy> ovl_by_dst(ovl_all.size());
  std::vector<int2> ovl_range(plist_all.size(), make_int2(0, 0));
  for (size_t li = 0; li < nl; ++li) {
    const int p0 = span_plist[li].first, np = span_plist[li].second;
    const int o0 = span_ovl[li].first, no = span_ovl[li].second;
    int at = o0;
    for (int k = 0; k < np; ++k) {
      const int dst = plist_all[p0 + k];
      const int first = at;
      for (int c = o0; c < o0 + no; ++c)
        if (ovl_all[c].dst == dst) ovl_by_dst[at++] = ovl_all[c];
      ovl_range[p0 + k] = make_int2(first - o0, at - first);
    }
    if (at != o0 + no) return fail(h, BSAM_ERR_ARG, "an overlap names no patch of its level");
  }
  h->h_plist = plist_all;
  h->h_ovl_by_dst = ovl_by_dst;
  h->h_ovl_range = ovl_range;
  h->h_span_plist = span_plist;
  h->h_span_ovl = span_ovl;
  h->max_items = std::max(1, h->nmaster);
  for (size_t li = 0; li < nl; ++li) {
    LevelPlan& L = h->levels[li];
    L.nplist = span_plist[li].second;
    L.novl = span_ovl[li].second;
    L.nfine = spans_fine[li].second;
    L.ncoarse = spans_coarse[li].second;
    L.nfused = spans_fused[li].second;
    h->max_items = std::max(h->max_items, L.nfine);
  }
  h->max_items = std::max(h->max_items, h->nroot);
  if (!h->attrs_set) {
    CU(cudaFuncSetAttribute(k_smooth3_fused<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)Fused3<double>::SMEM));
    CU(cudaFuncSetAttribute(k_smooth3_fused<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)Fused3<float>::SMEM));
    h->attrs_set = true;
  }
  // The residual trace buffers live as long as the handle (maxvcycles is
  // fixed at creation).
  if (!h->d_trace) CU(cudaMalloc(&h->d_trace, sizeof(double) * h->rp.maxvcycles));
  if (!h->h_trace) CU(cudaMallocHost(&h->h_trace, sizeof(double) * h->rp.maxvcycles));
  {
    int64_t ncells = 0;
    for (int p : h->masters) ncells += cells_of(h->hp[p].n, nd);
    h->denom = (double)(h->rp.nrvars * ncells);  // L2Error's integralresult(2)
  }
  std::vector<int> tops;
  if (h->bottom_level >= minlevel) {
    tops = plan(h, h->bottom_level).patches;
    for (int p : tops)
      if (h->hp[p].prec != PREC_F64) return fail(h, BSAM_ERR_ARG, "bottom levels must be FP64");
    h->ntops = (int)tops.size();
  }
  // The tables' layout in d_meta (256-byte aligned pieces), the buffer grown
  // when too small, then the pointers, and one copy of the host image.
  {
    size_t off = 0;
    auto place = [&](size_t bytes) {
      const size_t at = (size_t)roundup((int64_t)off, 256);
      off = at + bytes;
      return at;
    };
    const size_t o_patches = place(sizeof(DevPatch) * nrec);
    const size_t o_items = place(sizeof(Item) * all.size());
    const size_t o_plist = place(sizeof(int) * plist_all.size());
    const size_t o_ovl = place(sizeof(OverlapCopy) * ovl_all.size());
    const size_t o_ovl_dst = place(sizeof(OverlapCopy) * ovl_by_dst.size());
    const size_t o_ovl_rng = place(sizeof(int2) * ovl_range.size());
    const size_t o_qold = place(sizeof(CopySpan) * qold_spans.size());
    const size_t o_maps = place(sizeof(CUtensorMap) * maps.size());
    const size_t o_tops = place(sizeof(int) * tops.size());
    const size_t o_part = place(sizeof(double) * h->max_items);
    const size_t total_meta = off;
    if (total_meta > h->meta_cap) {
      if (h->d_meta) cudaFree(h->d_meta);
      h->d_meta = nullptr;
      h->meta_cap = 0;
      const size_t want = total_meta + total_meta / 2;  // headroom for the next regrid
      if (cudaMalloc(&h->d_meta, want) != cudaSuccess)
        return fail(h, BSAM_ERR_NOMEM, "table allocation failed");
      h->meta_cap = want;
    }
    char* base = h->d_meta;
    h->d_items = reinterpret_cast<Item*>(base + o_items);
    h->d_plist = plist_all.empty() ? nullptr : reinterpret_cast<int*>(base + o_plist);
    h->d_ovl = ovl_all.empty() ? nullptr : reinterpret_cast<OverlapCopy*>(base + o_ovl);
    h->d_qold_spans = qold_spans.empty() ? nullptr : reinterpret_cast<CopySpan*>(base + o_qold);
    h->d_tmaps = maps.empty() ? nullptr : reinterpret_cast<CUtensorMap*>(base + o_maps);
    h->d_tops = tops.empty() ? nullptr : reinterpret_cast<int*>(base + o_tops);
    h->d_partials = reinterpret_cast<double*>(base + o_part);
    h->d_patches = reinterpret_cast<DevPatch*>(base + o_patches);
    for (size_t k = 0; k < fused_recs.size(); ++k) h->hp[fused_recs[k]].tmaps = h->d_tmaps + 7 * k;
    for (size_t li = 0; li < nl; ++li) {
      LevelPlan& L = h->levels[li];
      L.d_plist = h->d_plist ? h->d_plist + span_plist[li].first : nullptr;
      L.d_ovl = h->d_ovl ? h->d_ovl + span_ovl[li].first : nullptr;
      L.d_ovl_by_dst = ovl_by_dst.empty()
                           ? nullptr
                           : reinterpret_cast<OverlapCopy*>(base + o_ovl_dst) + span_ovl[li].first;
      L.d_ovl_range = ovl_range.empty()
                          ? nullptr
                          : reinterpret_cast<int2*>(base + o_ovl_rng) + span_plist[li].first;
      L.d_fine = h->d_items + spans_fine[li].first;
      L.d_coarse = h->d_items + spans_coarse[li].first;
      L.d_fused = h->d_items + spans_fused[li].first;
    }
    h->d_master = h->d_items + s_master;
    h->d_state = h->d_items + s_state;
    h->d_root = h->d_items + s_root;
    std::vector<unsigned char>& img = h->meta_host;
    img.assign(o_part, 0);  // the partial sums need no initial contents
    auto put = [&](size_t at, const void* src, size_t bytes) {
      if (bytes) std::memcpy(img.data() + at, src, bytes);
    };
    put(o_patches, h->hp.data(), sizeof(DevPatch) * nrec);
    put(o_items, all.data(), sizeof(Item) * all.size());
    put(o_plist, plist_all.data(), sizeof(int) * plist_all.size());
    put(o_ovl, ovl_all.data(), sizeof(OverlapCopy) * ovl_all.size());
    put(o_ovl_dst, ovl_by_dst.data(), sizeof(OverlapCopy) * ovl_by_dst.size());
    put(o_ovl_rng, ovl_range.data(), sizeof(int2) * ovl_range.size());
    put(o_qold, qold_spans.data(), sizeof(CopySpan) * qold_spans.size());
    put(o_maps, maps.data(), sizeof(CUtensorMap) * maps.size());
    put(o_tops, tops.data(), sizeof(int) * tops.size());
    const int urc = h2d_bounce(h, h->d_meta, img.data(), img.size());
    if (urc) return urc;
  }
  CU(cudaMemsetAsync(h->d_status, 0, sizeof(DevStatus), h->stream));
  CU(cudaStreamSynchronize(h->stream));
  h->have_hierarchy = true;
  return BSAM_OK;
}

static int field_ptr(bsam_gpu* h, int patch, int field, int comp, double** ptr, bool* interior) {
  const DevPatch& P = h->hp[patch];
  void* p = nullptr;
  *interior = false;
  switch (field) {
    case BSAM_FIELD_Q: p = P.q[comp]; break;
    case BSAM_FIELD_QOLD: p = P.qo[comp]; break;
    case BSAM_FIELD_F: p = P.f[comp]; *interior = true; break;
    default: return BSAM_ERR_ARG;
  }
  if (!p) return BSAM_ERR_UNSUPPORTED;
  *ptr = static_cast<double*>(p);
  return BSAM_OK;
}

// Copy between a Fortran array and the pitched device field; dir 0 = H2D.
static int copy_field(bsam_gpu* h, int patch, int field, double* host, int dir) {
  if (!h || !h->have_hierarchy) return BSAM_ERR_STATE;
  if (patch < 0 || patch >= h->nuser || !host) return BSAM_ERR_ARG;
  CU(cudaSetDevice(h->device));
  const DevPatch& P = h->hp[patch];
  if (P.prec != PREC_F64 || P.delta)
    return fail(h, BSAM_ERR_UNSUPPORTED, "the fields of mixed-precision working levels are internal");
  const int nd = h->rp.ndims;
  for (int comp = 0; comp < 2; ++comp) {
    double* dev;
    bool interior;
    const int rc = field_ptr(h, patch, field, comp, &dev, &interior);
    if (rc) return fail(h, rc, "field not held for this patch");
    const int g = interior ? 0 : 1;  // ghost layers present in the host array
    const int e0 = P.n[0] + 2 * g, e1 = P.n[1] + 2 * g, e2 = nd == 3 ? P.n[2] + 2 * g : 1;
    const size_t hcomp = (size_t)e0 * e1 * e2;
    double* hbase = host + comp * hcomp;
    if (g == 1) {
      // With the ghost ring every row of every plane sits at stride sy on the
      // device (sz = sy * (n1 + 2)): one pitched copy per component.
      if (dir == 0)
        CU(cudaMemcpy2DAsync(dev, P.sy * sizeof(double), hbase, e0 * sizeof(double),
                             e0 * sizeof(double), (size_t)e1 * e2, cudaMemcpyHostToDevice,
                             h->stream));
      else
        CU(cudaMemcpy2DAsync(hbase, e0 * sizeof(double), dev, P.sy * sizeof(double),
                             e0 * sizeof(double), (size_t)e1 * e2, cudaMemcpyDeviceToHost,
                             h->stream));
      continue;
    }
    for (int kz = 0; kz < e2; ++kz) {
      const int k = nd == 3 ? kz + 1 : 0;
      double* d = dev + 1 + P.sy + (int64_t)k * P.sz;
      double* hs = hbase + (size_t)kz * e0 * e1;
      if (dir == 0)
        CU(cudaMemcpy2DAsync(d, P.sy * sizeof(double), hs, e0 * sizeof(double),
                             e0 * sizeof(double), e1, cudaMemcpyHostToDevice, h->stream));
      else
        CU(cudaMemcpy2DAsync(hs, e0 * sizeof(double), d, P.sy * sizeof(double),
                             e0 * sizeof(double), e1, cudaMemcpyDeviceToHost, h->stream));
    }
  }
  CU(cudaStreamSynchronize(h->stream));
  return BSAM_OK;
}

int bsam_gpu_put_field(bsam_gpu* h, int patch, int field, const double* a) {
  return copy_field(h, patch, field, const_cast<double*>(a), 0);
}

int bsam_gpu_get_field(bsam_gpu* h, int patch, int field, double* out) {
  return copy_field(h, patch, field, out, 1);
}

int bsam_gpu_set_ghost(bsam_gpu* h) {
  if (!h || !h->have_hierarchy) return BSAM_ERR_STATE;
  CU(cudaSetDevice(h->device));
  // Coarse levels first: a refined level's interpolation reads its parent.
  for (int l = h->minlevel; l <= h->finestlevel; ++l) {
    if (plan(h, l).amr) amr_ghost(h, l, 0);
    else ghost_level(h, l);
  }
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(h->stream));
  return BSAM_OK;
}

int bsam_gpu_set_ghost_level(bsam_gpu* h, int level) {
  if (!h || !h->have_hierarchy) return BSAM_ERR_STATE;
  if (level < h->minlevel || level > h->finestlevel)
    return fail(h, BSAM_ERR_ARG, "set_ghost_level: level out of range");
  CU(cudaSetDevice(h->device));
  if (plan(h, level).amr) amr_ghost(h, level, 0);
  else ghost_level(h, level);
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(h->stream));
  return BSAM_OK;
}

int bsam_gpu_fill_down(bsam_gpu* h) {
  if (!h || !h->have_hierarchy) return BSAM_ERR_STATE;
  CU(cudaSetDevice(h->device));
  if (h->amr) filldown(h);
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(h->stream));
  return BSAM_OK;
}

int bsam_gpu_restrict_level(bsam_gpu* h, int level) {
  if (!h || !h->have_hierarchy) return BSAM_ERR_STATE;
  if (level < 1 || level > h->finestlevel)
    return fail(h, BSAM_ERR_ARG, "restrict_level needs a refined level");
  CU(cudaSetDevice(h->device));
  const LevelPlan& L = plan(h, level);
  if (h->rp.ndims == 2)
    k_filldown<2><<<L.ncoarse, block_dim(), 0, h->stream>>>(h->d_patches, L.d_coarse);
  else
    k_filldown<3><<<L.ncoarse, block_dim(), 0, h->stream>>>(h->d_patches, L.d_coarse);
  ++h->stats.launches;
  amr_ghost(h, level - 1, 0);
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(h->stream));
  return BSAM_OK;
}

int bsam_gpu_copy_q_to_qold(bsam_gpu* h) {
  if (!h || !h->have_hierarchy) return BSAM_ERR_STATE;
  CU(cudaSetDevice(h->device));
  // qold exists on levels >= root only (Source reads it there).
  if (h->nqold_spans == 0) return BSAM_OK;
  const int bx = (int)std::min<int64_t>((h->qold_span_max + 255) / 256, 64);
  k_copy_spans<<<dim3(bx, h->nqold_spans), 256, 0, h->stream>>>(h->d_qold_spans);
  ++h->stats.launches;
  CU(cudaGetLastError());
  return BSAM_OK;
}

int bsam_gpu_multigrid_iterations(bsam_gpu* h, int* nvcycles, double* residual, int* converged) {
  if (!h || !h->have_hierarchy) return BSAM_ERR_STATE;
  CU(cudaSetDevice(h->device));
  const int nd = h->rp.ndims;
  const dim3 b = block_dim();
  // FillDown(solution) (afas:47) over the refined levels; below the root it
  // and FillDown(source) (afas:66, 90) only write regions that
  // RestrictSolution / CoarseLoadingFunction overwrite before any read, so
  // they are not issued.  Then GetSourceFunction + UpdateSourceFunction on
  // the state patches of levels >= root (afas:57-64).
  if (h->amr) filldown(h);
  if (nd == 2) k_source<double, 2><<<h->nstate, b, 0, h->stream>>>(h->d_patches, h->d_state);
  else k_source<double, 3><<<h->nstate, b, 0, h->stream>>>(h->d_patches, h->d_state);
  ++h->stats.launches;
  // Mixed form: the FP32 working copy and its right-hand side for the first
  // V-cycle (the norm computed here is not a convergence test).
  if (h->mixed) launch_resid(h);
  h->trace.clear();
  int it = 0, conv = 0;
  double res = 0.0;
  if (h->tuning.graph == 0 && !h->profiling) {
    // The whole V-cycle loop as one graph launch (device-side WHILE node).
    if (!h->step_exec) {
      const int rc = build_step_graph(h);
      if (rc) return rc;
    }
    k_mg_begin<<<1, 1, 0, h->stream>>>(h->d_status);
    CU(cudaGetLastError());
    CU(cudaGraphLaunch(h->step_exec, h->stream));
    CU(cudaMemcpyAsync(h->h_status, h->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost,
                       h->stream));
    CU(cudaMemcpyAsync(h->h_trace, h->d_trace, sizeof(double) * h->rp.maxvcycles,
                       cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    it = std::max(1, std::min(h->h_status->iters, h->rp.maxvcycles));
    h->stats.launches += 1 + (int64_t)h->graph_kernels_per_vcycle * h->h_status->iters;
    res = h->h_status->residual;
    h->trace.assign(h->h_trace, h->h_trace + it);
    if (nvcycles) *nvcycles = it;
    if (residual) *residual = res;
    if (converged) *converged = 0;
    if (h->h_status->kerr)
      return fail(h, BSAM_ERR_CUDA, "a fused smoothing stage timed out waiting for its copies");
    if (!std::isfinite(res)) return fail(h, BSAM_ERR_DIVERGED, "residual is not finite");
    if (converged) *converged = h->h_status->converged;
    return BSAM_OK;
  }
  for (it = 1; it <= h->rp.maxvcycles; ++it) {
    iteration(h);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(h->h_status, h->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost,
                       h->stream));
    CU(cudaStreamSynchronize(h->stream));
    drain_events(h);
    res = h->h_status->residual;
    if (h->h_status->kerr) {
      if (nvcycles) *nvcycles = it;
      if (residual) *residual = res;
      if (converged) *converged = 0;
      return fail(h, BSAM_ERR_CUDA, "a fused smoothing stage timed out waiting for its copies");
    }
    h->trace.push_back(res);
    if (!std::isfinite(res)) {
      if (nvcycles) *nvcycles = it;
      if (residual) *residual = res;
      if (converged) *converged = 0;
      return fail(h, BSAM_ERR_DIVERGED, "residual is not finite");
    }
    if (res < h->rp.qerrortol) {
      conv = 1;
      break;
    }
  }
  if (it > h->rp.maxvcycles) it = h->rp.maxvcycles;
  if (nvcycles) *nvcycles = it;
  if (residual) *residual = res;
  if (converged) *converged = conv;
  return BSAM_OK;
}

int bsam_gpu_residual_trace(bsam_gpu* h, double* out, int maxn) {
  if (!h) return BSAM_ERR_ARG;
  const int n = std::min<int>(maxn, (int)h->trace.size());
  for (int i = 0; i < n; ++i) out[i] = h->trace[i];
  return (int)h->trace.size();
}

int bsam_gpu_mass(bsam_gpu* h, double* mass) {
  if (!h || !h->have_hierarchy || !mass) return BSAM_ERR_STATE;
  if (h->nroot == 0) return fail(h, BSAM_ERR_UNSUPPORTED, "no root-level patch");
  CU(cudaSetDevice(h->device));
  // AfterStep2D/3D integral(1) on the root level (problem.f90:102-134).
  int root = 0;
  for (int p = 0; p < h->nuser; ++p)
    if (h->desc[p].level == 0) root = p;
  const double hh = h->hp[root].h;
  const double hd = h->rp.ndims == 2 ? hh * hh : hh * hh * hh;
  if (h->rp.ndims == 2)
    k_mass<double, 2><<<h->nroot, block_dim(), 0, h->stream>>>(
        h->d_patches, h->d_root, h->d_partials, h->d_status, h->nroot, hd);
  else
    k_mass<double, 3><<<h->nroot, block_dim(), 0, h->stream>>>(
        h->d_patches, h->d_root, h->d_partials, h->d_status, h->nroot, hd);
  ++h->stats.launches;
  CU(cudaGetLastError());
  CU(cudaMemcpyAsync(h->h_status, h->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost,
                     h->stream));
  CU(cudaStreamSynchronize(h->stream));
  *mass = h->h_status->mass;
  return BSAM_OK;
}

int bsam_gpu_errflags(bsam_gpu* h, int patch, double tol, uint8_t* flags) {
  if (!h || !h->have_hierarchy || !flags) return BSAM_ERR_ARG;
  if (patch < 0 || patch >= h->nuser || h->desc[patch].level < 0)
    return fail(h, BSAM_ERR_ARG, "errflags needs a patch on a level >= 0");
  CU(cudaSetDevice(h->device));
  const DevPatch& P = h->hp[patch];
  const int nd = h->rp.ndims;
  const size_t ncell = (size_t)P.n[0] * P.n[1] * (nd == 3 ? P.n[2] : 1);
  uint8_t* d_flags = nullptr;
  CU(cudaMalloc(&d_flags, ncell));
  const int blocks = (int)std::min<size_t>((ncell + 255) / 256, 4096);
  if (nd == 2) k_errflags<2><<<blocks, 256, 0, h->stream>>>(h->d_patches, patch, tol, d_flags);
  else k_errflags<3><<<blocks, 256, 0, h->stream>>>(h->d_patches, patch, tol, d_flags);
  ++h->stats.launches;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(flags, d_flags, ncell, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(d_flags);
  if (e != cudaSuccess) return fail(h, BSAM_ERR_CUDA, cudaGetErrorString(e));
  return BSAM_OK;
}

// Copies a host task list into the handle's task buffer (grown, never
// shrunk) on the stream; the caller synchronises before the next upload.
static int upload_tasks(bsam_gpu* h, const void* src, size_t bytes) {
  if (bytes > h->regrid_cap) {
    if (h->d_regrid) cudaFree(h->d_regrid);
    h->d_regrid = nullptr;
    h->regrid_cap = 0;
    const size_t want = bytes + bytes / 2;
    if (cudaMalloc(&h->d_regrid, want) != cudaSuccess)
      return fail(h, BSAM_ERR_NOMEM, "task buffer allocation failed");
    h->regrid_cap = want;
  }
  return h2d_bounce(h, h->d_regrid, src, bytes);
}

int bsam_gpu_errflags_level(bsam_gpu* h, int level, double tol, uint8_t* flags) {
  if (!h || !h->have_hierarchy || !flags) return BSAM_ERR_ARG;
  if (level < 0 || level > h->finestlevel)
    return fail(h, BSAM_ERR_ARG, "errflags_level needs a level >= 0");
  CU(cudaSetDevice(h->device));
  const int nd = h->rp.ndims;
  size_t total = 0;
  for (int p = 0; p < h->nuser; ++p)
    if (h->desc[p].level == level) total += (size_t)cells_of(h->hp[p].n, nd);
  if (total == 0) return BSAM_OK;
  if (total > h->flags_cap) {
    if (h->d_flags) cudaFree(h->d_flags);
    h->d_flags = nullptr;
    h->flags_cap = 0;
    if (cudaMalloc(&h->d_flags, total) != cudaSuccess)
      return fail(h, BSAM_ERR_NOMEM, "flag buffer allocation failed");
    h->flags_cap = total;
  }
  // One launch over the level: a task per patch (offset into the flags).
  std::vector<FlagTask> tasks;
  size_t off = 0, ncell_max = 0;
  for (int p = 0; p < h->nuser; ++p) {
    if (h->desc[p].level != level) continue;
    const size_t ncell = (size_t)cells_of(h->hp[p].n, nd);
    tasks.push_back(FlagTask{(int64_t)off, p, 0});
    ncell_max = std::max(ncell_max, ncell);
    off += ncell;
  }
  if (tasks.size() > 65535) return fail(h, BSAM_ERR_ARG, "errflags_level: too many patches");
  const int rc = upload_tasks(h, tasks.data(), sizeof(FlagTask) * tasks.size());
  if (rc) return rc;
  const dim3 g((unsigned)std::min<size_t>((ncell_max + 255) / 256, 1024), (unsigned)tasks.size());
  const FlagTask* d_tasks = reinterpret_cast<const FlagTask*>(h->d_regrid);
  if (nd == 2) k_errflags_list<2><<<g, 256, 0, h->stream>>>(h->d_patches, d_tasks, tol, h->d_flags);
  else k_errflags_list<3><<<g, 256, 0, h->stream>>>(h->d_patches, d_tasks, tol, h->d_flags);
  ++h->stats.launches;
  CU(cudaGetLastError());
  {
    const int drc = d2h_bounce(h, flags, h->d_flags, total);
    if (drc) return drc;
  }
  return BSAM_OK;
}

int bsam_gpu_tag_level(bsam_gpu* h, int level, double tol, int ibuffer, int32_t* sat) {
  if (!h || !h->have_hierarchy || !sat || ibuffer < 0) return BSAM_ERR_ARG;
  if (level < 0 || level > h->finestlevel)
    return fail(h, BSAM_ERR_ARG, "tag_level needs a level >= 0");
  CU(cudaSetDevice(h->device));
  const int nd = h->rp.ndims;
  // The level's patches in table order, their cells concatenated.
  std::vector<FlagTask> tasks;
  std::vector<LevelPatch> lp;
  size_t total = 0, ncell_max = 0;
  for (int p = 0; p < h->nuser; ++p) {
    if (h->desc[p].level != level) continue;
    const size_t ncell = (size_t)cells_of(h->hp[p].n, nd);
    tasks.push_back(FlagTask{(int64_t)total, p, 0});
    LevelPatch L{};
    L.off = (int64_t)total;
    for (int n = 0; n < 3; ++n) {
      L.n[n] = n < nd ? h->hp[p].n[n] : 1;
      L.g0[n] = n < nd ? h->desc[p].mglobal[n][0] : 1;
    }
    lp.push_back(L);
    ncell_max = std::max(ncell_max, ncell);
    total += ncell;
  }
  if (total == 0) return BSAM_OK;
  const int np = (int)tasks.size();
  if (np > 65535) return fail(h, BSAM_ERR_ARG, "tag_level: too many patches");
  if (2 * total > h->flags_cap) {
    if (h->d_flags) cudaFree(h->d_flags);
    h->d_flags = nullptr;
    h->flags_cap = 0;
    if (cudaMalloc(&h->d_flags, 2 * total) != cudaSuccess)
      return fail(h, BSAM_ERR_NOMEM, "flag buffer allocation failed");
    h->flags_cap = 2 * total;
  }
  if (total > h->sat_cap) {
    if (h->d_sat) cudaFree(h->d_sat);
    h->d_sat = nullptr;
    h->sat_cap = 0;
    if (cudaMalloc(&h->d_sat, sizeof(int32_t) * total) != cudaSuccess)
      return fail(h, BSAM_ERR_NOMEM, "summed-area table allocation failed");
    h->sat_cap = total;
  }
  // One upload: the tagging tasks, then the level's patches.
  std::vector<unsigned char> buf(sizeof(FlagTask) * np + sizeof(LevelPatch) * np);
  std::memcpy(buf.data(), tasks.data(), sizeof(FlagTask) * np);
  std::memcpy(buf.data() + sizeof(FlagTask) * np, lp.data(), sizeof(LevelPatch) * np);
  int rc = upload_tasks(h, buf.data(), buf.size());
  if (rc) return rc;
  const FlagTask* d_tasks = reinterpret_cast<const FlagTask*>(h->d_regrid);
  const LevelPatch* d_lp = reinterpret_cast<const LevelPatch*>(h->d_regrid + sizeof(FlagTask) * np);
  uint8_t* raw = h->d_flags;
  uint8_t* buffered = h->d_flags + total;
  const dim3 g((unsigned)std::min<size_t>((ncell_max + 255) / 256, 1024), (unsigned)np);
  if (nd == 2) {
    k_errflags_list<2><<<g, 256, 0, h->stream>>>(h->d_patches, d_tasks, tol, raw);
    k_buffer_list<2><<<g, 256, 0, h->stream>>>(d_lp, np, ibuffer, raw, buffered);
    k_sat_list<2><<<np, 256, 0, h->stream>>>(d_lp, buffered, h->d_sat);
  } else {
    k_errflags_list<3><<<g, 256, 0, h->stream>>>(h->d_patches, d_tasks, tol, raw);
    k_buffer_list<3><<<g, 256, 0, h->stream>>>(d_lp, np, ibuffer, raw, buffered);
    k_sat_list<3><<<np, 256, 0, h->stream>>>(d_lp, buffered, h->d_sat);
  }
  h->stats.launches += 3;
  CU(cudaGetLastError());
  return d2h_bounce(h, sat, h->d_sat, sizeof(int32_t) * total);
}

int bsam_gpu_init_patch(bsam_gpu* h, int patch) {
  if (!h || !h->have_hierarchy) return BSAM_ERR_ARG;
  if (patch < 0 || patch >= h->nuser || h->desc[patch].level < 1)
    return fail(h, BSAM_ERR_ARG, "init_patch needs a refined patch (level >= 1)");
  const DevPatch& P = h->hp[patch];
  if (!P.qo[0] || h->mixed) return fail(h, BSAM_ERR_UNSUPPORTED, "init_patch: FP64 form only");
  CU(cudaSetDevice(h->device));
  const int nd = h->rp.ndims;
  const size_t ncoarse = (size_t)(P.cn[0] + 2) * (P.cn[1] + 2) * (nd == 3 ? P.cn[2] + 2 : 1);
  const int blocks = (int)std::min<size_t>((ncoarse + 255) / 256, 4096);
  if (nd == 2) k_init_mc<2><<<blocks, 256, 0, h->stream>>>(h->d_patches, patch);
  else k_init_mc<3><<<blocks, 256, 0, h->stream>>>(h->d_patches, patch);
  ++h->stats.launches;
  CU(cudaGetLastError());
  return BSAM_OK;
}

int bsam_gpu_energy(bsam_gpu* h, double* energy) {
  if (!h || !h->have_hierarchy || !energy) return BSAM_ERR_STATE;
  if (h->rp.ndims != 2 || h->amr || h->nroot == 0)
    return fail(h, BSAM_ERR_UNSUPPORTED,
                "the energy is defined for a 2D hierarchy without refined levels (AfterStep2D "
                "at level 0)");
  CU(cudaSetDevice(h->device));
  int root = 0;
  for (int p = 0; p < h->nuser; ++p)
    if (h->desc[p].level == 0) root = p;
  const double hh = h->hp[root].h, h2 = hh * hh;
  const double tmp = h->rp.eps * h->rp.eps / h2 / 4.0;  // eps2/h2/4.0 (problem.f90:355)
  double s[2];
  for (int which = 0; which < 2; ++which) {
    k_energy2<double><<<h->nroot, block_dim(), 0, h->stream>>>(
        h->d_patches, h->d_root, h->d_partials, h->d_status, h->nroot, which);
    ++h->stats.launches;
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(h->h_status, h->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost,
                       h->stream));
    CU(cudaStreamSynchronize(h->stream));
    s[which] = h->h_status->esum;
  }
  *energy = h2 * (s[0] + tmp * s[1]);
  return BSAM_OK;
}

int bsam_gpu_after_step_stats(bsam_gpu* h, double* integral) {
  if (!h || !h->have_hierarchy || !integral) return BSAM_ERR_ARG;
  const int nd = h->rp.ndims;
  // The terms, in the order AfterStepStatistics adds them: levels finest to
  // root, ApplyOnLevel (table) order within a level.  Per patch: sum(c), then
  // (2D) Ff and squared-difference sums; on a refined patch the same over its
  // parent's footprint.
  struct Term {
    int patch, kind, lo[3], hi[3];
  };
  std::vector<Term> terms;
  std::vector<int> order;
  for (int level = h->finestlevel; level >= 0; --level)
    for (int p = 0; p < h->nuser; ++p)
      if (h->desc[p].level == level) order.push_back(p);
  for (int p : order) {
    const bsam_patch_desc& d = h->desc[p];
    if (h->hp[p].prec != PREC_F64) return fail(h, BSAM_ERR_UNSUPPORTED, "stats need FP64 patches");
    const int nk = nd == 2 ? 3 : 1;  // 2D adds the two energy sums
    for (int side = 0; side < (d.level > 0 ? 2 : 1); ++side) {
      Term t{};
      t.patch = side == 0 ? p : d.parent;
      if (side == 1 && h->hp[t.patch].prec != PREC_F64)
        return fail(h, BSAM_ERR_UNSUPPORTED, "stats need FP64 patches");
      for (int n = 0; n < 3; ++n) {
        if (n >= nd) {
          t.lo[n] = t.hi[n] = 0;
        } else if (side == 0) {
          t.lo[n] = 1;
          t.hi[n] = d.mx[n];
        } else {
          t.lo[n] = d.mbounds[n][0];
          t.hi[n] = d.mbounds[n][1];
        }
      }
      for (int kind = 0; kind < nk; ++kind) {
        t.kind = kind;
        terms.push_back(t);
      }
    }
  }
  // Split each term's rows over CTAs (about 16k cells a CTA).
  std::vector<StatBlock> blocks;
  std::vector<int> first(terms.size() + 1, 0);
  for (size_t ti = 0; ti < terms.size(); ++ti) {
    const Term& t = terms[ti];
    const int nx = t.hi[0] - t.lo[0] + 1, ny = t.hi[1] - t.lo[1] + 1;
    const int nz = nd == 3 ? t.hi[2] - t.lo[2] + 1 : 1;
    const int rows = ny * nz;
    const int per = std::max(1, 16384 / std::max(1, nx));
    first[ti] = (int)blocks.size();
    for (int r0 = 0; r0 < rows; r0 += per) {
      StatBlock b{};
      b.patch = t.patch;
      b.kind = t.kind;
      for (int n = 0; n < 3; ++n) {
        b.lo[n] = t.lo[n];
        b.hi[n] = t.hi[n];
      }
      b.row0 = r0;
      b.row1 = std::min(rows, r0 + per);
      blocks.push_back(b);
    }
  }
  first[terms.size()] = (int)blocks.size();
  const int nb = (int)blocks.size();
  CU(cudaSetDevice(h->device));
  StatBlock* d_blocks = nullptr;
  double* d_part = nullptr;
  std::vector<double> part(nb);
  cudaError_t e = cudaMalloc(&d_blocks, sizeof(StatBlock) * nb);
  if (e == cudaSuccess) e = cudaMalloc(&d_part, sizeof(double) * nb);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_blocks, blocks.data(), sizeof(StatBlock) * nb, cudaMemcpyHostToDevice,
                        h->stream);
  if (e == cudaSuccess) {
    if (nd == 2) k_stats<2><<<nb, 256, 0, h->stream>>>(h->d_patches, d_blocks, d_part);
    else k_stats<3><<<nb, 256, 0, h->stream>>>(h->d_patches, d_blocks, d_part);
    ++h->stats.launches;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(part.data(), d_part, sizeof(double) * nb, cudaMemcpyDeviceToHost,
                        h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (d_blocks) cudaFree(d_blocks);
  if (d_part) cudaFree(d_part);
  if (e != cudaSuccess) return fail(h, BSAM_ERR_CUDA, cudaGetErrorString(e));
  auto term_sum = [&](size_t ti) {
    double s = 0.0;
    for (int b = first[ti]; b < first[ti + 1]; ++b) s += part[b];
    return s;
  };
  // Combine as AfterStep2D/3D do.
  const double eps2 = h->rp.eps * h->rp.eps;
  double r1 = 0.0, r2 = 0.0;
  size_t ti = 0;
  auto energy = [&](double hh, double sF, double sG) {
    const double h2 = hh * hh;
    return h2 * (sF + eps2 / h2 / 4.0 * sG);
  };
  for (int p : order) {
    const bsam_patch_desc& d = h->desc[p];
    const double hh = h->hp[p].h, ch = hh * 2.0;
    const double hd = nd == 2 ? hh * hh : hh * hh * hh;
    const double chd = nd == 2 ? ch * ch : ch * ch * ch;
    if (nd == 2) {
      const double s = term_sum(ti), sF = term_sum(ti + 1), sG = term_sum(ti + 2);
      ti += 3;
      if (d.level == 0) {
        r1 = r1 + hd * s;
        r2 = r2 + energy(hh, sF, sG);
      } else {
        const double cs = term_sum(ti), cF = term_sum(ti + 1), cG = term_sum(ti + 2);
        ti += 3;
        r1 = r1 + hd * s - chd * cs;
        r2 = r2 + energy(hh, sF, sG) - energy(ch, cF, cG);
      }
    } else {
      const double s = term_sum(ti);
      ti += 1;
      if (d.level == 0) {
        r1 = r1 + hd * s;
      } else {
        const double cs = term_sum(ti);
        ti += 1;
        r1 = r1 + hd * s - chd * cs;
      }
    }
  }
  integral[0] = r1;
  integral[1] = r2;
  return BSAM_OK;
}

int bsam_gpu_stash(bsam_gpu* h) {
  if (!h || !h->have_hierarchy) return BSAM_ERR_STATE;
  if (h->mixed) return fail(h, BSAM_ERR_UNSUPPORTED, "regridding: FP64 form only");
  CU(cudaSetDevice(h->device));
  h->stash_hp.assign(h->nuser, DevPatch{});
  h->stash_desc = h->desc;
  size_t total = 0;
  std::vector<size_t> off(h->nuser, 0);
  for (int p = 0; p < h->nuser; ++p)
    if (h->desc[p].level >= 1) {
      off[p] = total;
      total += 2 * (size_t)h->field_elems[p] * sizeof(double);
    }
  if (total == 0) return BSAM_OK;
  if (total > h->stash_cap) {
    if (h->d_stash) cudaFree(h->d_stash);
    h->d_stash = nullptr;
    h->stash_cap = 0;
    const size_t want = total + total / 2;  // headroom for the next steps
    if (cudaMalloc(&h->d_stash, want) != cudaSuccess)
      return fail(h, BSAM_ERR_NOMEM, "stash allocation failed");
    h->stash_cap = want;
  }
  const int64_t lead = 128 / sizeof(double) - 1;
  std::vector<CopySpan> spans;
  int64_t span_max = 0;
  for (int p = 0; p < h->nuser; ++p) {
    if (h->desc[p].level < 1) continue;
    DevPatch S = h->hp[p];
    for (int c = 0; c < 2; ++c) {
      double* dst = reinterpret_cast<double*>(h->d_stash + off[p]) + c * h->field_elems[p];
      spans.push_back(CopySpan{static_cast<const double*>(S.q[c]) - lead, dst, h->field_elems[p]});
      S.q[c] = dst + lead;
    }
    span_max = std::max(span_max, h->field_elems[p]);
    h->stash_hp[p] = S;
  }
  if (spans.size() > h->stash_spans_cap) {
    if (h->d_stash_spans) cudaFree(h->d_stash_spans);
    h->d_stash_spans = nullptr;
    h->stash_spans_cap = 0;
    const size_t want = spans.size() + spans.size() / 2;
    if (cudaMalloc(&h->d_stash_spans, sizeof(CopySpan) * want) != cudaSuccess)
      return fail(h, BSAM_ERR_NOMEM, "stash allocation failed");
    h->stash_spans_cap = want;
  }
  {
    const int urc = h2d_bounce(h, h->d_stash_spans, spans.data(), sizeof(CopySpan) * spans.size());
    if (urc) return urc;
  }
  const int bx = (int)std::min<int64_t>((span_max + 255) / 256, 64);
  k_copy_spans<<<dim3(bx, (unsigned)spans.size()), 256, 0, h->stream>>>(h->d_stash_spans);
  ++h->stats.launches;
  CU(cudaGetLastError());
  // The span list is host memory: wait until it has been read.
  CU(cudaStreamSynchronize(h->stream));
  return BSAM_OK;
}

int bsam_gpu_regrid(bsam_gpu* h, int npatch, const bsam_patch_desc* patches, int finestlevel,
                    const int* carry, int ntransfer, const int* transfer) {
  if (!h || !h->have_hierarchy || npatch <= 0 || !patches || !carry || ntransfer < 0 ||
      (ntransfer > 0 && !transfer))
    return BSAM_ERR_ARG;
  if (h->mixed) return fail(h, BSAM_ERR_UNSUPPORTED, "regridding: FP64 form only");
  const int nd = h->rp.ndims;
  const int nold = h->nuser;
  for (int i = 0; i < npatch; ++i) {
    const int o = carry[i];
    if (o < -1 || o >= nold) return fail(h, BSAM_ERR_ARG, "regrid: carry index out of range");
    if (o >= 0) {
      if (h->desc[o].level != patches[i].level)
        return fail(h, BSAM_ERR_ARG, "regrid: a carried patch changes level");
      for (int n = 0; n < nd; ++n)
        if (h->desc[o].mx[n] != patches[i].mx[n])
          return fail(h, BSAM_ERR_ARG, "regrid: a carried patch changes size");
    } else if (patches[i].level < 1) {
      return fail(h, BSAM_ERR_ARG, "regrid: only refined patches may be new");
    }
  }
  for (int t = 0; t < ntransfer; ++t) {
    const int c = transfer[2 * t], s = transfer[2 * t + 1];
    if (c < 0 || c >= npatch || carry[c] >= 0 || s < 0 || s >= (int)h->stash_hp.size() ||
        h->stash_desc[s].level != patches[c].level)
      return fail(h, BSAM_ERR_ARG, "regrid: a transfer names no new grid and stashed grid");
  }
  CU(cudaSetDevice(h->device));
  CU(cudaStreamSynchronize(h->stream));
  // Keep the old arena (the carried q and qold) until the copies are done.
  char* old_arena = h->d_arena;
  const size_t old_bytes = h->arena_bytes;
  h->d_arena = nullptr;
  const std::vector<DevPatch> old_hp = h->hp;
  const std::vector<int64_t> old_fe = h->field_elems;
  h->regridding = true;
  int rc = bsam_gpu_set_hierarchy(h, npatch, patches, finestlevel);
  h->regridding = false;
  if (rc != BSAM_OK) {
    cudaFree(old_arena);
    return rc;
  }
  // The device work as three launches from one uploaded task list: the
  // carried patches' q and qold (whole field allocations), InitFields of every
  // new grid from its carried parent, then the transfers from the stash.
  const int64_t lead = 128 / sizeof(double) - 1;
  cudaError_t e = cudaSuccess;
  std::vector<CopySpan> spans;
  std::vector<int> children;
  std::vector<TransferTask> tasks;
  int64_t span_max = 0, child_max = 0, task_max = 0;
  for (int i = 0; i < npatch; ++i) {
    const int o = carry[i];
    if (o < 0) {
      const DevPatch& P = h->hp[i];
      children.push_back(i);
      child_max = std::max<int64_t>(
          child_max, (int64_t)(P.cn[0] + 2) * (P.cn[1] + 2) * (nd == 3 ? P.cn[2] + 2 : 1));
      continue;
    }
    const DevPatch& A = old_hp[o];
    const DevPatch& B = h->hp[i];
    if (old_fe[o] != h->field_elems[i]) {
      e = cudaErrorInvalidValue;
      break;
    }
    for (int c = 0; c < 2; ++c) {
      spans.push_back(CopySpan{static_cast<const double*>(A.q[c]) - lead,
                               static_cast<double*>(B.q[c]) - lead, old_fe[o]});
      if (A.qo[c] && B.qo[c])
        spans.push_back(CopySpan{static_cast<const double*>(A.qo[c]) - lead,
                                 static_cast<double*>(B.qo[c]) - lead, old_fe[o]});
    }
    span_max = std::max(span_max, old_fe[o]);
  }
  for (int t = 0; t < ntransfer && e == cudaSuccess; ++t) {
    const int c = transfer[2 * t], s = transfer[2 * t + 1];
    const bsam_patch_desc& T = patches[c];
    const bsam_patch_desc& S = h->stash_desc[s];
    TransferTask tk{};
    tk.S = h->stash_hp[s];
    tk.target = c;
    bool empty = false;
    int64_t cells = 1;
    for (int n = 0; n < 3; ++n) {
      if (n >= nd) {
        tk.n[n] = 1;
        continue;
      }
      const int lo = std::max(T.mglobal[n][0], S.mglobal[n][0]);
      const int hi = std::min(T.mglobal[n][1], S.mglobal[n][1]);
      empty |= hi < lo;
      tk.n[n] = hi - lo + 1;
      tk.si[n] = lo - S.mglobal[n][0] + 1;
      tk.ti[n] = lo - T.mglobal[n][0] + 1;
      cells *= tk.n[n];
    }
    if (empty) continue;
    tasks.push_back(tk);
    task_max = std::max(task_max, cells);
  }
  if (e == cudaSuccess && (spans.size() > 65535 || children.size() > 65535 || tasks.size() > 65535))
    e = cudaErrorInvalidValue;  // one grid row per item: at most 65535 of each
  if (e == cudaSuccess && (!spans.empty() || !children.empty() || !tasks.empty())) {
    // Layout: spans, children, tasks; 256-byte aligned pieces.
    const size_t o_sp = 0;
    const size_t o_ch = (size_t)roundup((int64_t)(sizeof(CopySpan) * spans.size()), 256);
    const size_t o_tk = o_ch + (size_t)roundup((int64_t)(sizeof(int) * children.size()), 256);
    const size_t bytes = o_tk + sizeof(TransferTask) * tasks.size();
    h->regrid_host.assign(bytes, 0);
    unsigned char* img = h->regrid_host.data();
    if (!spans.empty()) std::memcpy(img + o_sp, spans.data(), sizeof(CopySpan) * spans.size());
    if (!children.empty()) std::memcpy(img + o_ch, children.data(), sizeof(int) * children.size());
    if (!tasks.empty()) std::memcpy(img + o_tk, tasks.data(), sizeof(TransferTask) * tasks.size());
    const int urc = upload_tasks(h, img, bytes);
    if (urc != BSAM_OK) {
      cudaFree(old_arena);
      return urc;
    }
    const auto grid_x = [](int64_t n) { return (unsigned)std::min<int64_t>((n + 255) / 256, 64); };
    if (e == cudaSuccess && !spans.empty()) {
      k_copy_spans<<<dim3(grid_x(span_max), (unsigned)spans.size()), 256, 0, h->stream>>>(
          reinterpret_cast<const CopySpan*>(h->d_regrid + o_sp));
      ++h->stats.launches;
      e = cudaGetLastError();
    }
    if (e == cudaSuccess && !children.empty()) {
      const dim3 g(grid_x(child_max), (unsigned)children.size());
      const int* d_ch = reinterpret_cast<const int*>(h->d_regrid + o_ch);
      if (nd == 2) k_init_mc_list<2><<<g, 256, 0, h->stream>>>(h->d_patches, d_ch);
      else k_init_mc_list<3><<<g, 256, 0, h->stream>>>(h->d_patches, d_ch);
      ++h->stats.launches;
      e = cudaGetLastError();
    }
    if (e == cudaSuccess && !tasks.empty()) {
      const dim3 g(grid_x(task_max), (unsigned)tasks.size());
      const TransferTask* d_tk = reinterpret_cast<const TransferTask*>(h->d_regrid + o_tk);
      if (nd == 2) k_transfer_list<2><<<g, 256, 0, h->stream>>>(h->d_patches, d_tk);
      else k_transfer_list<3><<<g, 256, 0, h->stream>>>(h->d_patches, d_tk);
      ++h->stats.launches;
      e = cudaGetLastError();
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  // The old arena becomes the spare (the larger of it and the current spare).
  if (h->spare_arena && h->spare_bytes >= old_bytes) {
    cudaFree(old_arena);
  } else {
    if (h->spare_arena) cudaFree(h->spare_arena);
    h->spare_arena = old_arena;
    h->spare_bytes = old_bytes;
  }
  if (e != cudaSuccess) return fail(h, BSAM_ERR_CUDA, cudaGetErrorString(e));
  return BSAM_OK;
}

int bsam_gpu_set_tuning(bsam_gpu* h, const bsam_tuning* t) {
  if (!h || !t) return BSAM_ERR_ARG;
  if (t->fuse_smoother < -1 || t->fuse_smoother > 1 || t->chunk < 0 || t->graph < -1 ||
      t->graph > 0)
    return BSAM_ERR_ARG;
  h->tuning = *t;
  if (h->step_exec) {
    cudaGraphExecDestroy(h->step_exec);
    h->step_exec = nullptr;
  }
  return BSAM_OK;
}

int bsam_gpu_get_stream(bsam_gpu* h, void** stream) {
  if (!h || !stream) return BSAM_ERR_ARG;
  *stream = (void*)h->stream;
  return BSAM_OK;
}

int bsam_gpu_profile(bsam_gpu* h, int enable) {
  if (!h) return BSAM_ERR_ARG;
  if (enable) {
    h->stats = bsam_gpu_stats{};
    h->ev_used = 0;
    if (h->have_hierarchy) {
      h->ev_cells = 0;
      const LevelPlan& F = plan(h, h->finestlevel);
      for (int p : F.patches) h->ev_cells += cells_of(h->hp[p].n, h->rp.ndims);
      h->ev_bytes = elem_bytes(F.prec);
    }
  }
  h->profiling = enable != 0;
  return BSAM_OK;
}

int bsam_gpu_get_stats(bsam_gpu* h, bsam_gpu_stats* out) {
  if (!h || !out) return BSAM_ERR_ARG;
  if (h->ev_used) {
    cudaStreamSynchronize(h->stream);
    drain_events(h);
  }
  *out = h->stats;
  return BSAM_OK;
}

int bsam_gpu_destroy(bsam_gpu* h) {
  if (!h) return BSAM_ERR_ARG;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (auto& e : h->ev_pool) {
    cudaEventDestroy(e.first);
    cudaEventDestroy(e.second);
  }
  free_hierarchy(h);
  if (h->d_trace) cudaFree(h->d_trace);
  if (h->h_trace) cudaFreeHost(h->h_trace);
  if (h->h_pin) cudaFreeHost(h->h_pin);
  if (h->spare_arena) cudaFree(h->spare_arena);
  if (h->d_stash) cudaFree(h->d_stash);
  if (h->d_stash_spans) cudaFree(h->d_stash_spans);
  if (h->d_meta) cudaFree(h->d_meta);
  if (h->d_regrid) cudaFree(h->d_regrid);
  if (h->d_flags) cudaFree(h->d_flags);
  if (h->d_sat) cudaFree(h->d_sat);
  if (h->d_status) cudaFree(h->d_status);
  if (h->h_status) cudaFreeHost(h->h_status);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return BSAM_OK;
}

}  // extern "C"
