// bsam_batch.cu -- C ABI of the batched / continuously batched engine
// (include/bsam_batch.h).
//
// Device state of a batch:
//  * one memory pool; each resident problem ("slot") holds one contiguous
//    region of it with all its fields, laid out exactly as bsam_gpu.cu lays
//    out a single problem (pitched SoA, 128-byte aligned interior rows);
//  * one patch table with a fixed block of RMAX records per slot;
//  * work lists (Items) per V-cycle stage and depth, shared by all slots and
//    appended to on admission; their lengths live on the device;
//  * per-slot configuration / state / step log, and a mapped host mirror of
//    each slot's phase that the host polls without synchronising.
// A tick (one V-cycle of every running problem + its control) is captured
// once into a graph whose WHILE node repeats ticks on the device; the graph
// is captured again only when a list outgrows its capacity or a problem with
// more grid-kernel depths arrives.
//
// Records of one slot (local index): FP64 form 0 = root (level 0), l =
// level -l; mixed form 0 = FP64 master, 1 = working twin of the root,
// l + 1 = level -l.  Depth d of the V-cycle is level -d.  Depths whose
// levels have more than bottom_cells cells run grid kernels ("top" depths);
// the rest run inside the bottom kernel's chain, as in the single-problem
// engine with the same bottom_cells, and are FP64 in both forms.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "../../include/bsam_batch.h"
#include "batch.cuh"
#include "bsam_types.h"
#include "defect2.cuh"
#include "engine_view.h"
#include "fused2.cuh"

using namespace bsam;

namespace {

constexpr int RMAX = 16;  // records per slot
constexpr int NMAPS = 7;  // TMA maps per fused record
constexpr int MAXD = 8;   // top depths
// Default bottom_cells: levels of at most this many cells run in the bottom
// kernel (in FP64 in both forms, as bsam_gpu.cu does with the same value).
constexpr int DEFAULT_BOTTOM_CELLS = 1024;
// Default runs of consecutive list entries per CTA visit (TileRuns) for the
// small-tile list kernels and for the fused stages (tuning.tile_chunk and
// tuning.fused_chunk; 1 = grid-stride order).
constexpr int kDefaultTileChunk = 2;
constexpr int kDefaultFusedChunk = 1;
// Runs of the staged defect, in units of tile_chunk.
constexpr int kDefectRunFactor = 4;
// Lists: master tiles; bottom-chain tops; per top depth d: tiles of every
// record (correction), footprint tiles (restriction / coarse load), tiles of
// records smoothed per colour pass, fused-stage tiles; master tiles whose FP64
// update is not done by their post-smoothing stage (mixed form, finest
// working level not fused).
enum {
  L_MASTER = 0,
  L_TOPS = 1,
  L_FINE = 2,
  L_COARSE = 2 + MAXD,
  L_RELAX = 2 + 2 * MAXD,
  L_FUSED = 2 + 3 * MAXD,
  L_CORR = 2 + 4 * MAXD,  // 2D: tiles of 2 x 2 fine-cell blocks (kb_correct2)
  L_UPD = 2 + 5 * MAXD,
  L_RESTR = 3 + 5 * MAXD,  // footprint tiles of records restricted by kb_restrict
  NLIST = 3 + 6 * MAXD
};

// Lists of the refined hierarchies (SLOT_AMR), over the records of their own
// table: finest-level tiles (ErrorAFAS), bottom-chain tops; per depth d (up
// to MAXD, the depth below the last top one included): interior tiles
// (colour passes, correction), footprint tiles (restriction, coarse load),
// footprint tiles of refined records (FillDown), refined records with their
// GhostOverlap transfers (SetGhost), rows of partly covered parents
// (snapshot).
enum {
  A_MASTER = 0,
  A_TOPS = 1,
  A_FINE = 2,
  A_COARSE = 2 + (MAXD + 1),
  A_FILL = 2 + 2 * (MAXD + 1),
  A_GHOST = 2 + 3 * (MAXD + 1),
  A_SNAP = 2 + 4 * (MAXD + 1),
  A_RELAX = 2 + 5 * (MAXD + 1),  // 2D: colour-pass tiles shaped to the patch width
  ANLIST = 2 + 6 * (MAXD + 1)
};

struct List {
  Item* d = nullptr;
  int cap = 0;            // device capacity in items
  std::vector<Item> h;
  int uploaded = 0;       // h[0, uploaded) are on the device
};

struct SlotPlan {
  bool used = false;
  bool stale = false;     // retired, and its tiles are still in the lists
  size_t off = 0, bytes = 0;
  int nrec = 0, ntop = 0, master = 0, top = 0;
  int64_t cells = 0;
  bsam_batch_problem prob{};
  std::vector<DevPatch> recs;  // absolute record indices
  std::vector<CUtensorMap> maps;  // NMAPS per record (fused records only encoded)
  // A refined hierarchy (bsam_batch_submit_amr): its driver and engine, the
  // engine's current hierarchy, and where its records start in the refined
  // hierarchies' table.
  bool amr = false;
  bsam_amr* drv = nullptr;
  bsam_gpu* eng = nullptr;
  EngineView view;
  int arec0 = 0, chain = 0, nsteps = 0;
  cudaEvent_t ready = nullptr;  // the engine's regrid and prologue are done
};

struct StageChunk {
  size_t a, b;
  cudaEvent_t ev;
};

int64_t roundup(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

int64_t cells_of(const int* n, int nd) {
  int64_t c = 1;
  for (int d = 0; d < nd; ++d) c *= n[d];
  return c;
}

void tiles_for(int patch, const int* n, int nd, std::vector<Item>& out) {
  const int tx = (n[0] + TILE_X - 1) / TILE_X;
  const int ty = (n[1] + TILE_Y - 1) / TILE_Y;
  const int tz = nd == 3 ? n[2] : 1;
  for (int z = 0; z < tz; ++z)
    for (int y = 0; y < ty; ++y)
      for (int x = 0; x < tx; ++x) out.push_back(Item{patch, x, y, z});
}

}  // namespace

struct bsam_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  bsam_batch_params bp{};
  bool mixed = false;
  int nsm = 148;
  bsam_batch_tuning tuning{};
  // pool
  char* d_pool = nullptr;
  size_t pool_bytes = 0, pool_used = 0;
  std::map<size_t, size_t> free_;  // offset -> size, coalesced
  // records, slots
  DevPatch* d_pt = nullptr;
  CUtensorMap* d_tmaps = nullptr;  // NMAPS per record: fused stages' TMA maps
  std::vector<SlotPlan> slots;
  SlotCfg* d_cfg = nullptr;
  std::vector<SlotCfg> h_cfg;
  bool cfg_dirty = false;
  SlotState* d_state = nullptr;
  StepLog* d_log = nullptr;
  SlotOut* h_out = nullptr;  // mapped
  SlotOut* d_out = nullptr;
  BatchCtl* d_ctl = nullptr;
  DevStatus* d_status = nullptr;
  DevStatus* h_status = nullptr;
  double* d_partials = nullptr;
  int partials_cap = 0;
  List lists[NLIST];
  int* d_counts = nullptr;
  std::vector<int> counts_dev;  // counts last uploaded
  // Refined hierarchies: their records, transfers and lists (append-only;
  // retired entries stay inactive until amr_compact rebuilds them).
  std::vector<DevPatch> h_apt;
  DevPatch* d_apt = nullptr;
  int apt_cap = 0, apt_uploaded = 0;
  std::vector<OverlapCopy> h_aovl;
  OverlapCopy* d_aovl = nullptr;
  int aovl_cap = 0, aovl_uploaded = 0;
  List alists[ANLIST];
  int* d_acounts = nullptr;
  std::vector<int> acounts_dev;
  double* d_apartials = nullptr;
  int apartials_cap = 0;
  // graph
  cudaGraphExec_t exec = nullptr;
  int cap_depth = 0;
  bool need_capture = true;
  int64_t kernels_per_tick = 0;
  bsam_batch_stats st{};
  // profiling (eager ticks): events around the finest-depth smoothing stages
  bool profiling = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pool;
  std::vector<char> ev_post;  // per timed stage: post-smoothing (dir 1)
  size_t ev_used = 0;
  // pinned staging ring for host -> device copies
  char* stage = nullptr;
  size_t stage_bytes = 0, stage_head = 0;
  std::deque<StageChunk> chunks;
  std::vector<size_t> pending;  // chunk indices (into `chunks`) awaiting an event
  std::vector<cudaEvent_t> free_events;
  // Device transfer buffers of the batched submit (in) and collect (out):
  // packed root states between the caller's buffers and the pitched fields.
  // The submitted states are copied in on their own stream, so that the
  // copies overlap ticks already queued on `stream`: xin_ready (copy stream)
  // orders the spreading launch after them, xin_free (engine stream) orders
  // the next copies after that launch.
  double* d_xin = nullptr;
  size_t xin_words = 0;
  double* d_xout = nullptr;
  size_t xout_words = 0;
  cudaStream_t xstream = nullptr;
  cudaEvent_t xin_ready = nullptr, xin_free = nullptr;
  std::string err;
};

namespace {

int fail(bsam_batch* b, int code, const std::string& msg) {
  if (b) b->err = msg;
  return code;
}

#define CU(call)                                                                  \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess)                                                        \
      return fail(b, BSAM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// ---- pool ----------------------------------------------------------------------

bool pool_alloc(bsam_batch* b, size_t bytes, size_t* off) {
  for (auto it = b->free_.begin(); it != b->free_.end(); ++it) {
    if (it->second < bytes) continue;
    *off = it->first;
    const size_t rest = it->second - bytes, at = it->first + bytes;
    b->free_.erase(it);
    if (rest) b->free_[at] = rest;
    b->pool_used += bytes;
    return true;
  }
  return false;
}

void pool_free(bsam_batch* b, size_t off, size_t bytes) {
  auto it = b->free_.emplace(off, bytes).first;
  auto nx = std::next(it);
  if (nx != b->free_.end() && it->first + it->second == nx->first) {
    it->second += nx->second;
    b->free_.erase(nx);
  }
  if (it != b->free_.begin()) {
    auto pv = std::prev(it);
    if (pv->first + pv->second == it->first) {
      pv->second += it->second;
      b->free_.erase(it);
    }
  }
  b->pool_used -= bytes;
}

// ---- staging ring ------------------------------------------------------------

cudaEvent_t take_event(bsam_batch* b) {
  if (!b->free_events.empty()) {
    cudaEvent_t e = b->free_events.back();
    b->free_events.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  return e;
}

// Marks every chunk staged since the last call as done once the work queued
// so far on `st` (the engine's stream by default) has executed.
void stage_commit(bsam_batch* b, cudaStream_t st = nullptr) {
  if (b->pending.empty()) return;
  cudaEvent_t e = take_event(b);
  cudaEventRecord(e, st ? st : b->stream);
  for (size_t i : b->pending) b->chunks[i].ev = e;
  b->pending.clear();
}

// Pinned host memory for n bytes, valid until the copies queued from it have
// executed (stage_commit).
char* stage_alloc(bsam_batch* b, size_t n) {
  n = (size_t)roundup((int64_t)std::max<size_t>(n, 1), 256);
  if (n > b->stage_bytes) {
    // Grow: wait for everything staged so far, then replace the ring.
    cudaStreamSynchronize(b->stream);
    for (auto& c : b->chunks)
      if (c.ev && std::find(b->free_events.begin(), b->free_events.end(), c.ev) ==
                      b->free_events.end())
        b->free_events.push_back(c.ev);
    b->chunks.clear();
    b->pending.clear();
    if (b->stage) cudaFreeHost(b->stage);
    b->stage_bytes = std::max({n, 2 * b->stage_bytes, (size_t)64 << 20});
    if (cudaMallocHost(&b->stage, b->stage_bytes) != cudaSuccess) {
      b->stage = nullptr;
      b->stage_bytes = 0;
      return nullptr;
    }
    b->stage_head = 0;
  }
  if (b->stage_head + n > b->stage_bytes) b->stage_head = 0;
  const size_t a = b->stage_head, e = a + n;
  // Chunks are in allocation order; the ones this range overlaps are at the
  // front (the previous lap of the ring).
  while (!b->chunks.empty()) {
    StageChunk& c = b->chunks.front();
    if (c.b <= a || c.a >= e) break;
    if (!c.ev) stage_commit(b);  // staged in this call sequence: fence it now
    cudaEventSynchronize(c.ev);
    // The event may be shared with later chunks: recycle it with the last.
    const cudaEvent_t ev = c.ev;
    b->chunks.pop_front();
    for (size_t& i : b->pending) --i;
    bool shared = false;
    for (auto& o : b->chunks) shared |= o.ev == ev;
    if (!shared) b->free_events.push_back(ev);
  }
  b->chunks.push_back(StageChunk{a, e, nullptr});
  b->pending.push_back(b->chunks.size() - 1);
  b->stage_head = e;
  return b->stage + a;
}

// Queues a host -> device copy of n bytes through the staging ring.
int stage_copy(bsam_batch* b, void* dst, const void* src, size_t n) {
  char* s = stage_alloc(b, n);
  if (!s) return fail(b, BSAM_ERR_NOMEM, "pinned staging allocation failed");
  std::memcpy(s, src, n);
  CU(cudaMemcpyAsync(dst, s, n, cudaMemcpyHostToDevice, b->stream));
  return BSAM_OK;
}

// A device transfer buffer with room for `words` doubles (grown after the
// work queued on both streams has drained); nullptr if the allocation fails.
double* xfer_reserve(bsam_batch* b, double** buf, size_t* have, size_t words) {
  if (words > *have) {
    if (*buf) {
      cudaStreamSynchronize(b->stream);
      cudaStreamSynchronize(b->xstream);
      cudaFree(*buf);
      *buf = nullptr;
    }
    const size_t w = std::max(words, 2 * *have);
    if (cudaMalloc(buf, sizeof(double) * w) != cudaSuccess) {
      *buf = nullptr;
      *have = 0;
      return nullptr;
    }
    *have = w;
  }
  return *buf;
}

// ---- problem plan ----------------------------------------------------------------

int face_rule(int nd, int face, int code, int* rule) {
  if (code == 1) *rule = BC_COPY;
  else if (code >= 10 && code <= 99) *rule = (nd == 2 && face >= 2) ? BC_COPY : BC_REFLECT;
  else return -1;  // internal faces and periodic faces have no batch form
  return 0;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda).
PFN_cuTensorMapEncodeTiled_v12000 map_encoder() {
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

// 2D map of one field of a 2D record: rows of sy elements from the
// allocation start (lead elements before element (0,0)), n1 + 2 rows, box
// bx x by (default: the fused stage's shared tile, RX x RY).
bool encode_map2d(CUtensorMap* m, const DevPatch& P, const void* field, int bx = 0, int by = 0) {
  auto enc = map_encoder();
  if (!enc) return false;
  const bool f32 = P.prec == PREC_F32;
  const int es = f32 ? 4 : 8;
  const int64_t lead = 128 / es - 1;
  void* base = (char*)field - lead * es;
  const cuuint64_t dims[2] = {(cuuint64_t)P.sy, (cuuint64_t)(P.n[1] + 2)};
  const cuuint64_t strides[1] = {(cuuint64_t)(P.sy * es)};
  if (bx == 0) {
    bx = f32 ? Fused2<float>::RX : Fused2<double>::RX;
    by = f32 ? Fused2<float>::RY : Fused2<double>::RY;
  }
  const cuuint32_t box[2] = {(cuuint32_t)bx, (cuuint32_t)by};
  const cuuint32_t estr[2] = {1, 1};
  return enc(m, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, base,
             dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Builds the slot's records (absolute indices from rec0; field pointers
// relative to a pool region starting at `base`).  base == nullptr: size only.
int plan_slot(bsam_batch* b, const bsam_batch_problem* pr, int rec0, char* base, SlotPlan& S) {
  const int nd = b->bp.ndims;
  if (pr->grid.ndims != nd) return fail(b, BSAM_ERR_ARG, "problem ndims differs from the batch");
  if (pr->nsteps < 1 || pr->nsteps > BSAM_BATCH_MAX_STEPS)
    return fail(b, BSAM_ERR_ARG, "nsteps out of range");
  if (!(pr->dt > 0) || !(pr->eps > 0)) return fail(b, BSAM_ERR_ARG, "dt and eps must be positive");
  bsam_patch_desc desc[RMAX];
  int np = 0;
  int rc = bsam_host_build_uniform(&pr->grid, desc, RMAX - 1, &np);
  if (rc) return fail(b, rc, "grid rejected (see bsam_host_build_uniform)");
  const bool mixed = b->mixed;
  const int nrec = np + (mixed ? 1 : 0);
  // Depth of the first bottom level.
  int ntop = np;
  const int64_t bcells = b->bp.bottom_cells;
  for (int l = 0; l < np; ++l)
    if (cells_of(desc[l].mx, nd) <= bcells) {
      ntop = l;
      break;
    }
  if (ntop >= np)
    return fail(b, BSAM_ERR_UNSUPPORTED, "the coarsest level exceeds the bottom kernel's size");
  if (ntop > MAXD) return fail(b, BSAM_ERR_UNSUPPORTED, "too many levels above the bottom");
  if (np - ntop > BOTTOM_MAX_DEPTH) return fail(b, BSAM_ERR_UNSUPPORTED, "bottom chain too deep");
  auto rec_of = [&](int l) { return mixed ? (l == 0 ? 1 : l + 1) : l; };  // V-cycle record
  S.recs.assign(nrec, DevPatch{});
  S.maps.clear();
  S.nrec = nrec;
  S.ntop = ntop;
  S.master = 0;
  S.top = rec0 + rec_of(ntop);
  S.cells = cells_of(desc[0].mx, nd);
  const double eps2 = pr->eps * pr->eps;
  size_t total = 0;
  for (int r = 0; r < nrec; ++r) {
    const bool is_master_only = mixed && r == 0;
    const int l = mixed ? (r == 0 ? 0 : r - 1) : r;  // level index (desc)
    const bsam_patch_desc& d = desc[l];
    DevPatch& P = S.recs[r];
    P.ndims = nd;
    for (int n = 0; n < 3; ++n) P.n[n] = n < nd ? d.mx[n] : 1;
    P.parent = d.parent >= 0 ? rec0 + rec_of(d.parent) : -1;
    P.level = d.level;
    P.problem = rec0 / RMAX;
    P.active = 1;
    P.newstep = (r == 0) ? 1 : 0;
    P.twin = is_master_only ? rec0 + 1 : -1;
    P.master = (mixed && r == 1) ? rec0 : -1;
    const int64_t ncell = cells_of(P.n, nd);
    P.prec = (!mixed || is_master_only || ncell <= bcells) ? PREC_F64 : PREC_F32;
    for (int n = 0; n < 3; ++n) {
      P.cn[n] = 1;
      P.off[n] = 0;
    }
    if (d.parent >= 0)
      for (int n = 0; n < nd; ++n) {
        P.cn[n] = P.n[n] / 2;
        P.off[n] = d.mbounds[n][0] - 1;
      }
    P.wt = 1;
    for (int f = 0; f < 6; ++f) {
      if (f >= 2 * nd) {
        P.bc[f] = BC_NONE;
        continue;
      }
      int rule;
      if (face_rule(nd, f, d.mthbc[f], &rule))
        return fail(b, BSAM_ERR_UNSUPPORTED, "batch problems need physical faces (codes 1, 10-99)");
      P.bc[f] = rule;
      P.code[f] = d.mthbc[f];
    }
    P.delta = (mixed && !is_master_only) ? 1 : 0;
    if (P.delta)
      for (int f = 0; f < 2 * nd; ++f)
        if (P.bc[f] == BC_REFLECT) P.bc[f] = BC_NEGATE;
    // Fused shared-memory stages: 2D levels above the bottom, 2*nu <= 4.
    const int depth = mixed ? r - 1 : r;
    P.fused = (!b->tuning.per_pass && nd == 2 && !is_master_only && depth < ntop &&
               b->bp.nsmoothingpasses <= 2)
                  ? 1
                  : 0;
    P.zchunk = 1;
    const int es = P.prec == PREC_F32 ? 4 : 8;
    const int64_t A = 128 / es, lead = A - 1;
    P.sy = roundup(lead + P.n[0] + 2, A);
    P.sz = nd == 3 ? P.sy * (P.n[1] + 2) : 0;
    const int64_t vol = nd == 3 ? P.sz * (P.n[2] + 2) : P.sy * (P.n[1] + 2);
    const int64_t fe = roundup(lead + vol + 64, 256 / es);
    // Every V-cycle record below the root is the parent of the next finer
    // one and keeps the snapshot qs of its restricted state.
    const bool is_parent = !is_master_only && l >= 1;
    const int nfield = 4 + (is_parent ? 2 : 0) + (P.delta ? 1 : 0) + (P.fused ? 2 : 0);
    if (base) {
      char* rb = base + total;
      int slotn = 0;
      auto next = [&]() { return (void*)(rb + (fe * (slotn++) + lead) * es); };
      P.q[0] = next();
      P.q[1] = next();
      P.f[0] = next();
      P.f[1] = next();
      P.qo[0] = P.qo[1] = nullptr;  // the source reads q at the start of a step
      P.qs[0] = P.qs[1] = nullptr;
      if (is_parent) {
        P.qs[0] = next();
        P.qs[1] = next();
      }
      P.qb[0] = P.qb[1] = nullptr;
      P.bs = P.delta ? next() : nullptr;
      if (P.fused) {
        P.qb[0] = next();
        P.qb[1] = next();
      }
      P.tmaps = nullptr;
      if (P.fused) {
        // TMA maps of q0, q1, qb0, qb1, f0, f1, bs for the fused stage.
        if (S.maps.size() < (size_t)nrec * NMAPS) S.maps.assign((size_t)nrec * NMAPS, CUtensorMap{});
        const void* fields[NMAPS] = {P.q[0], P.q[1], P.qb[0], P.qb[1],
                                     P.f[0], P.f[1], P.bs ? P.bs : P.q[0]};
        for (int m = 0; m < NMAPS; ++m)
          if (!encode_map2d(&S.maps[(size_t)r * NMAPS + m], P, fields[m]))
            return fail(b, BSAM_ERR_CUDA, "cuTensorMapEncodeTiled rejected a field map");
        P.tmaps = b->d_tmaps + (size_t)(rec0 + r) * NMAPS;
      }
      if (is_master_only && nd == 2) {
        // The defect's staged tiles (kb_defect_tma): q0, q1 with a one-cell
        // halo, f0, f1.
        if (S.maps.size() < (size_t)nrec * NMAPS) S.maps.assign((size_t)nrec * NMAPS, CUtensorMap{});
        const void* fields[4] = {P.q[0], P.q[1], P.f[0], P.f[1]};
        for (int m = 0; m < 4; ++m) {
          const int bx = m < 2 ? Defect2::QX : Defect2::TX, by = m < 2 ? Defect2::QY : Defect2::TY;
          if (!encode_map2d(&S.maps[(size_t)r * NMAPS + m], P, fields[m], bx, by))
            return fail(b, BSAM_ERR_CUDA, "cuTensorMapEncodeTiled rejected a field map");
        }
        P.tmaps = b->d_tmaps + (size_t)(rec0 + r) * NMAPS;
      }
    }
    total += (size_t)fe * nfield * es;
    P.h = d.dx;
    const double h2 = d.dx * d.dx;
    P.dt = pr->dt;
    P.eps2 = eps2;
    P.alpha = pr->alpha;
    P.tmp1 = pr->dt / h2;
    P.tmp2 = eps2 / h2;
    P.tmp3 = (2.0 * nd) * eps2 / h2;
  }
  for (int r = 0; r < nrec; ++r) {
    DevPatch& P = S.recs[r];
    P.pprec = P.parent >= 0 ? S.recs[P.parent - rec0].prec : P.prec;
  }
  S.bytes = (size_t)roundup((int64_t)total, 4096);
  S.prob = *pr;
  return BSAM_OK;
}

// Appends a slot's tiles to the lists and records its master range.
void append_items(bsam_batch* b, int s) {
  SlotPlan& S = b->slots[s];
  const int nd = b->bp.ndims;
  const int rec0 = s * RMAX;
  SlotCfg& C = b->h_cfg[s];
  C.ib = (int)b->lists[L_MASTER].h.size();
  tiles_for(rec0 + S.master, S.recs[S.master].n, nd, b->lists[L_MASTER].h);
  C.ie = (int)b->lists[L_MASTER].h.size();
  if (b->mixed && !S.recs[1].fused)
    tiles_for(rec0 + S.master, S.recs[S.master].n, nd, b->lists[L_UPD].h);
  b->lists[L_TOPS].h.push_back(Item{S.top, 0, 0, 0});
  const int first = b->mixed ? 1 : 0;  // record of depth 0
  for (int d = 0; d < S.ntop; ++d) {
    const int r = first + d;
    const DevPatch& P = S.recs[r];
    tiles_for(rec0 + r, P.n, nd, b->lists[L_FINE + d].h);
    tiles_for(rec0 + r, P.cn, nd, b->lists[L_COARSE + d].h);
    // A 2D fused record's restriction is done by its pre-smoothing stage.
    if (!(nd == 2 && P.fused)) tiles_for(rec0 + r, P.cn, nd, b->lists[L_RESTR + d].h);
    if (!P.fused) {
      tiles_for(rec0 + r, P.n, nd, b->lists[L_RELAX + d].h);
    } else {
      const int tx = P.prec == PREC_F32 ? Fused2<float>::TX : Fused2<double>::TX;
      const int ty = P.prec == PREC_F32 ? Fused2<float>::TY : Fused2<double>::TY;
      for (int y = 0; y < (P.n[1] + ty - 1) / ty; ++y)
        for (int x = 0; x < (P.n[0] + tx - 1) / tx; ++x)
          b->lists[L_FUSED + d].h.push_back(Item{rec0 + r, x, y, 0});
    }
    // blocks (m, n), m = 0..cn0, n = 0..cn1, 32 x TILE_Y per tile; a fused
    // record's correction is applied by its post-smoothing stage instead.
    if (nd == 2 && !P.fused)
      for (int y = 0; y < (P.cn[1] + 1 + TILE_Y - 1) / TILE_Y; ++y)
        for (int x = 0; x < (P.cn[0] + 1 + 31) / 32; ++x)
          b->lists[L_CORR + d].h.push_back(Item{rec0 + r, x, y, 0});
  }
  b->cfg_dirty = true;
}

// Rebuilds every list from the resident slots (drops retired slots' tiles).
void compact(bsam_batch* b) {
  for (auto& L : b->lists) {
    L.h.clear();
    L.uploaded = 0;
  }
  for (size_t s = 0; s < b->slots.size(); ++s) {
    b->slots[s].stale = false;
    if (b->slots[s].used && !b->slots[s].amr) append_items(b, (int)s);
  }
  b->cfg_dirty = true;
}

// ---- refined hierarchies ------------------------------------------------------

// Depth layout of a refined hierarchy (its engine's current one, S.view):
// the levels above the first root-chain level of at most bottom_cells cells
// run list kernels at depths 0 .. ntop - 1 (depth = finestlevel - level);
// that level heads the problem's bottom chain.
int amr_plan(bsam_batch* b, SlotPlan& S) {
  const EngineView& V = S.view;
  const int nd = b->bp.ndims;
  if (V.mixed) return fail(b, BSAM_ERR_UNSUPPORTED, "refined hierarchies run in FP64");
  if (V.ndims != nd) return fail(b, BSAM_ERR_ARG, "problem ndims differs from the batch");
  if (V.nsmoothingpasses != b->bp.nsmoothingpasses)
    return fail(b, BSAM_ERR_ARG, "nsmoothingpasses differs from the batch's");
  if (V.masters.empty() || V.levels.empty()) return fail(b, BSAM_ERR_STATE, "empty hierarchy");
  int chain = V.minlevel - 1;
  for (int l = 0; l >= V.minlevel; --l) {
    const EngineLevelView& E = V.levels[l - V.minlevel];
    if (E.patches.size() != 1)
      return fail(b, BSAM_ERR_UNSUPPORTED, "levels at and below the root must be one patch");
    if (cells_of(V.recs[E.patches[0]].n, nd) <= b->bp.bottom_cells) {
      chain = l;
      break;
    }
  }
  if (chain < V.minlevel)
    return fail(b, BSAM_ERR_UNSUPPORTED, "the coarsest level exceeds the bottom kernel's size");
  if (V.finestlevel - chain > MAXD)
    return fail(b, BSAM_ERR_UNSUPPORTED, "too many levels above the bottom");
  if (chain - V.minlevel + 1 > BOTTOM_MAX_DEPTH)
    return fail(b, BSAM_ERR_UNSUPPORTED, "bottom chain too deep");
  S.chain = chain;
  S.ntop = V.finestlevel - chain;
  return BSAM_OK;
}

// Appends the records, transfers and tiles of refined slot s (S.view) and
// points its configuration at them; active: the records run from the next
// tick on.
void amr_append(bsam_batch* b, int s, bool active) {
  SlotPlan& S = b->slots[s];
  const EngineView& V = S.view;
  const int nd = b->bp.ndims;
  const int r0 = (int)b->h_apt.size();
  S.arec0 = r0;
  for (DevPatch P : V.recs) {
    if (P.parent >= 0) P.parent += r0;
    P.problem = s;
    P.active = active ? 1 : 0;
    P.fused = 0;  // colour passes one launch each; q holds the state throughout
    P.newstep = 0;
    P.tmaps = nullptr;
    P.twin = P.master = -1;
    P.qb[0] = P.qb[1] = nullptr;
    b->h_apt.push_back(P);
  }
  List* LA = b->alists;
  SlotCfg& C = b->h_cfg[s];
  C.kind = SLOT_AMR;
  C.rec0 = r0;
  C.nrec = (int)V.recs.size();
  C.master = r0 + V.masters[0];
  C.nsteps = S.nsteps;
  C.maxv = V.maxvcycles;
  C.denom = V.denom;
  C.tol = V.qerrortol;
  C.ib = (int)LA[A_MASTER].h.size();
  for (int p : V.masters) tiles_for(r0 + p, V.recs[p].n, nd, LA[A_MASTER].h);
  C.ie = (int)LA[A_MASTER].h.size();
  LA[A_TOPS].h.push_back(Item{r0 + V.levels[S.chain - V.minlevel].patches[0], 0, 0, 0});
  for (int l = V.finestlevel; l >= S.chain; --l) {
    const EngineLevelView& E = V.levels[l - V.minlevel];
    const int d = V.finestlevel - l;
    if (l > S.chain) {
      const int ob = (int)b->h_aovl.size();
      if (E.amr)
        for (OverlapCopy o : E.ovl) {
          o.dst += r0;
          o.src += r0;
          b->h_aovl.push_back(o);
        }
      for (size_t k = 0; k < E.patches.size(); ++k) {
        const int p = E.patches[k];
        const DevPatch& P = V.recs[p];
        tiles_for(r0 + p, P.n, nd, LA[A_FINE + d].h);
        if (nd == 2) {
          // W lanes per row: the narrowest of 8, 16, 32 whose 2W columns
          // cover the patch (or 32).
          const int W = P.n[0] <= 16 ? 8 : (P.n[0] <= 32 ? 16 : 32);
          const int rows = BLOCK_THREADS / W;
          for (int y = 0; y < (P.n[1] + rows - 1) / rows; ++y)
            for (int x = 0; x < (P.n[0] + 2 * W - 1) / (2 * W); ++x)
              LA[A_RELAX + d].h.push_back(Item{r0 + p, x, y, W});
        }
        tiles_for(r0 + p, P.cn, nd, LA[A_COARSE + d].h);
        if (E.amr) {
          tiles_for(r0 + p, P.cn, nd, LA[A_FILL + d].h);
          const int2 rg = k < E.range.size() ? E.range[k] : make_int2(0, 0);
          LA[A_GHOST + d].h.push_back(Item{r0 + p, ob + rg.x, rg.y, 0});
        }
      }
    }
    // Parents their children do not cover: qs = q after the restriction
    // into them (and their SetGhost), before the coarse load reads it.
    if (E.snap)
      for (int p : E.patches) {
        const DevPatch& P = V.recs[p];
        if (!P.qs[0]) continue;
        const int nk = nd == 3 ? P.n[2] + 2 : 1;
        for (int k = 0; k < nk; ++k)
          for (int j = 0; j < P.n[1] + 2; ++j) LA[A_SNAP + d].h.push_back(Item{r0 + p, 0, j, k});
      }
  }
  b->cfg_dirty = true;
}

// Rebuilds the refined hierarchies' table, transfers and lists from the
// resident refined slots that have records (waits for the stream: the
// mirrored phases are then exact, and only running slots' records are
// active).  Everything is uploaded again by the next flush.
int amr_compact(bsam_batch* b) {
  CU(cudaStreamSynchronize(b->stream));
  b->h_apt.clear();
  b->h_aovl.clear();
  for (auto& L : b->alists) {
    L.h.clear();
    L.uploaded = 0;
  }
  b->apt_uploaded = 0;
  b->aovl_uploaded = 0;
  for (size_t s = 0; s < b->slots.size(); ++s) {
    SlotPlan& S = b->slots[s];
    if (!S.used || !S.amr || S.view.recs.empty()) continue;
    if (((volatile SlotOut*)b->h_out)[s].phase != SLOT_RUNNING) continue;
    amr_append(b, (int)s, true);
  }
  return BSAM_OK;
}

int live_amr_records(bsam_batch* b) {
  int n = 0;
  for (auto& S : b->slots)
    if (S.used && S.amr) n += (int)S.view.recs.size();
  return n;
}

// Uploads the refined hierarchies' growth (records, transfers, lists,
// counts); storage that must grow is reallocated after a compaction, and
// the tick graph is captured again.
int amr_flush(bsam_batch* b) {
  if ((int)b->h_apt.size() > b->apt_cap || (int)b->h_aovl.size() > b->aovl_cap) {
    int rc = amr_compact(b);
    if (rc) return rc;
    if ((int)b->h_apt.size() > b->apt_cap) {
      if (b->d_apt) cudaFree(b->d_apt);
      b->d_apt = nullptr;
      int cap = std::max(1024, 2 * b->apt_cap);
      while (cap < (int)b->h_apt.size()) cap *= 2;
      if (cudaMalloc(&b->d_apt, sizeof(DevPatch) * cap) != cudaSuccess) {
        b->apt_cap = 0;
        return fail(b, BSAM_ERR_NOMEM, "record table allocation failed");
      }
      b->apt_cap = cap;
      b->need_capture = true;
    }
    if ((int)b->h_aovl.size() > b->aovl_cap) {
      if (b->d_aovl) cudaFree(b->d_aovl);
      b->d_aovl = nullptr;
      int cap = std::max(1024, 2 * b->aovl_cap);
      while (cap < (int)b->h_aovl.size()) cap *= 2;
      if (cudaMalloc(&b->d_aovl, sizeof(OverlapCopy) * cap) != cudaSuccess) {
        b->aovl_cap = 0;
        return fail(b, BSAM_ERR_NOMEM, "transfer table allocation failed");
      }
      b->aovl_cap = cap;
      b->need_capture = true;
    }
  }
  const int na = (int)b->h_apt.size();
  if (b->apt_uploaded < na) {
    const int rc = stage_copy(b, b->d_apt + b->apt_uploaded, b->h_apt.data() + b->apt_uploaded,
                              sizeof(DevPatch) * (na - b->apt_uploaded));
    if (rc) return rc;
    b->apt_uploaded = na;
  }
  const int no = (int)b->h_aovl.size();
  if (b->aovl_uploaded < no) {
    const int rc = stage_copy(b, b->d_aovl + b->aovl_uploaded, b->h_aovl.data() + b->aovl_uploaded,
                              sizeof(OverlapCopy) * (no - b->aovl_uploaded));
    if (rc) return rc;
    b->aovl_uploaded = no;
  }
  for (int l = 0; l < ANLIST; ++l) {
    List& L = b->alists[l];
    const int n = (int)L.h.size();
    if (n > L.cap) {
      CU(cudaStreamSynchronize(b->stream));
      if (L.d) cudaFree(L.d);
      L.d = nullptr;
      int cap = std::max(256, L.cap);
      while (cap < n) cap *= 2;
      if (cudaMalloc(&L.d, sizeof(Item) * cap) != cudaSuccess) {
        L.cap = 0;
        return fail(b, BSAM_ERR_NOMEM, "work list allocation failed");
      }
      L.cap = cap;
      L.uploaded = 0;
      b->need_capture = true;
      if (l == A_MASTER && cap > b->apartials_cap) {
        if (b->d_apartials) cudaFree(b->d_apartials);
        b->d_apartials = nullptr;
        if (cudaMalloc(&b->d_apartials, sizeof(double) * cap) != cudaSuccess)
          return fail(b, BSAM_ERR_NOMEM, "partials allocation failed");
        b->apartials_cap = cap;
      }
    }
    if (L.uploaded < n) {
      const int rc = stage_copy(b, L.d + L.uploaded, L.h.data() + L.uploaded,
                                sizeof(Item) * (n - L.uploaded));
      if (rc) return rc;
      L.uploaded = n;
    }
  }
  std::vector<int> counts(ANLIST);
  for (int l = 0; l < ANLIST; ++l) counts[l] = (int)b->alists[l].h.size();
  if (counts != b->acounts_dev) {
    const int rc = stage_copy(b, b->d_acounts, counts.data(), sizeof(int) * ANLIST);
    if (rc) return rc;
    b->acounts_dev = counts;
  }
  return BSAM_OK;
}

// ---- tick -------------------------------------------------------------------

int grid_for(bsam_batch* b, int l) {
  const int cap = std::max(1, b->lists[l].cap);
  const int lim = b->tuning.grid_ctas > 0 ? b->tuning.grid_ctas : 16 * b->nsm;
  return std::max(1, std::min(cap, lim));
}

void stage_mark(bsam_batch* b, int d, bool begin, int dir) {
  if (!b->profiling || d != 0) return;
  if (begin) {
    if (b->ev_used == b->ev_pool.size()) {
      cudaEvent_t x, y;
      cudaEventCreate(&x);
      cudaEventCreate(&y);
      b->ev_pool.push_back({x, y});
      b->ev_post.push_back(0);
    }
    b->ev_post[b->ev_used] = (char)dir;
    cudaEventRecord(b->ev_pool[b->ev_used].first, b->stream);
  } else {
    cudaEventRecord(b->ev_pool[b->ev_used].second, b->stream);
    ++b->ev_used;
  }
}

// Issues one tick.  in_graph: captured into the WHILE body (handle valid).
template <int D>
void tick_t(bsam_batch* b, cudaGraphConditionalHandle handle, int in_graph) {
  const dim3 blk(32, TILE_Y, 1);
  cudaStream_t s = b->stream;
  const int nu = b->bp.nsmoothingpasses;
  DevPatch* pt = b->d_pt;
  const int* cnt = b->d_counts;
  const List* L = b->lists;
  int64_t n = 0;
  // The order in which CTAs take list entries (runs of consecutive tiles).
  const TileRuns R{b->tuning.tile_chunk > 0 ? b->tuning.tile_chunk : kDefaultTileChunk};
  const TileRuns RF{b->tuning.fused_chunk > 0 ? b->tuning.fused_chunk : kDefaultFusedChunk};
  // The staged defect reuses a patch's records along a run: longer runs.
  const TileRuns RD{kDefectRunFactor * R.chunk};
  // Refined hierarchies: their own table, transfers and lists (FP64).
  DevPatch* apt = b->d_apt;
  const int* acnt = b->d_acounts;
  const List* LA = b->alists;
  const int gthreads = D == 2 ? 128 : 256;
  auto agrid = [&](int l) {
    const int cap = std::max(1, LA[l].cap);
    const int lim = b->tuning.grid_ctas > 0 ? b->tuning.grid_ctas : 16 * b->nsm;
    return std::max(1, std::min(cap, lim));
  };
  // SetGhost(level, ipass) of the refined records at depth d.
  auto aghost = [&](int d, int ipass) {
    if (d > MAXD || LA[A_GHOST + d].cap == 0) return;
    kb_ghost<D><<<agrid(A_GHOST + d), gthreads, 0, s>>>(apt, LA[A_GHOST + d].d,
                                                        acnt + A_GHOST + d, b->d_aovl, ipass);
    ++n;
  };
  // LevelRelax of the refined hierarchies' records at depth d: each colour
  // pass, then SetGhost of the refined ones (afas:536-545).
  auto arelax = [&](int d) {
    if (LA[A_FINE + d].cap == 0) return;
    for (int pass = 0; pass < nu; ++pass)
      for (int color = 0; color < 2; ++color) {
        if (D == 2)
          kb_relax_narrow2<<<agrid(A_RELAX + d), blk, 0, s>>>(apt, LA[A_RELAX + d].d,
                                                              acnt + A_RELAX + d, color, R);
        else
          kb_relax<double, D><<<agrid(A_FINE + d), blk, 0, s>>>(apt, LA[A_FINE + d].d,
                                                                acnt + A_FINE + d, color, R);
        ++n;
        aghost(d, color + 1);
      }
  };
  // LevelRelax of depth d for every running problem; dir selects the fused
  // stage's buffers (0: q -> qb before the correction, 1: qb -> q after).
  auto relax = [&](int d, int dir) {
    stage_mark(b, d, true, dir);
    if (L[L_RELAX + d].cap > 0)
      for (int pass = 0; pass < nu; ++pass)
        for (int color = 0; color < 2; ++color) {
          const int g = grid_for(b, L_RELAX + d);
          if (b->mixed)
            kb_relax<float, D><<<g, blk, 0, s>>>(pt, L[L_RELAX + d].d, cnt + L_RELAX + d, color,
                                                 R);
          else
            kb_relax<double, D><<<g, blk, 0, s>>>(pt, L[L_RELAX + d].d, cnt + L_RELAX + d, color,
                                                  R);
          ++n;
        }
    if (D == 2 && L[L_FUSED + d].cap > 0) {
      const int lim = b->tuning.fused_ctas > 0 ? b->tuning.fused_ctas : 4 * b->nsm;
      const int g = std::max(1, std::min(L[L_FUSED + d].cap, lim));
      // Every fused record of a mixed batch is a correction-form FP32 level;
      // of an FP64 batch, a plain FP64 level.  The finest working level's
      // post-smoothing applies the FP64 update (kb_update skips those masters).
      const int upd = (b->mixed && d == 0 && dir == 1) ? 1 : 0;
      // The build picked by fused_occ: 2 = two tile buffers per CTA (two
      // CTAs per SM), 3 / 4 = one buffer and that many CTAs per SM.
      const int occ = b->tuning.fused_occ;
      const int nbuf = occ == 2 ? 2 : 1;
      if (b->mixed) {
        auto k = occ == 2   ? kb_smooth2<float, true, 2, 2>
                 : occ == 3 ? kb_smooth2<float, true, 3>
                            : kb_smooth2<float, true, 4>;
        k<<<g, Fused2<float>::THREADS, nbuf * Fused2<float>::smem(true), s>>>(
            pt, L[L_FUSED + d].d, cnt + L_FUSED + d, dir, nu, upd, dir, 1 - dir,
            &b->d_ctl->kerr, RF);
      } else {
        auto k = occ == 2   ? kb_smooth2<double, false, 2, 2>
                 : occ == 3 ? kb_smooth2<double, false, 3>
                            : kb_smooth2<double, false, 4>;
        k<<<g, Fused2<double>::THREADS, nbuf * Fused2<double>::smem(false), s>>>(
            pt, L[L_FUSED + d].d, cnt + L_FUSED + d, dir, nu, 0, dir, 1 - dir,
            &b->d_ctl->kerr, RF);
      }
      ++n;
    }
    stage_mark(b, d, false, dir);
  };
  const int gm = grid_for(b, L_MASTER);
  // The mixed form's FP64 defect: 2D masters through staged tiles
  // (defect2.cuh), 3D ones directly (same values either way).
  auto launch_defect = [&](int newstep_only) {
    if (D == 2)
      kb_defect_tma<2><<<gm, blk, Defect2::SMEM, s>>>(pt, L[L_MASTER].d, cnt + L_MASTER,
                                                      b->d_partials, newstep_only,
                                                      &b->d_ctl->kerr, RD);
    else
      kb_defect<D><<<gm, blk, 0, s>>>(pt, L[L_MASTER].d, cnt + L_MASTER, b->d_partials,
                                      newstep_only, R);
  };
  kb_source<D><<<gm, blk, 0, s>>>(pt, L[L_MASTER].d, cnt + L_MASTER, R);
  ++n;
  if (b->mixed) {
    launch_defect(1);
    ++n;
  }
  for (int d = 0; d < b->cap_depth; ++d) {
    relax(d, 0);
    arelax(d);
    if (LA[A_COARSE + d].cap > 0) {
      // RestrictSolution, SetGhost of a refined parent level, the snapshot
      // of partly covered parents, CoarseLoadingFunction (afas:503-509).
      kb_restrict<double, D><<<agrid(A_COARSE + d), blk, 0, s>>>(apt, LA[A_COARSE + d].d,
                                                                 acnt + A_COARSE + d, R);
      ++n;
      aghost(d + 1, 0);
      if (LA[A_SNAP + d + 1].cap > 0) {
        kb_snap<D><<<agrid(A_SNAP + d + 1), blk, 0, s>>>(apt, LA[A_SNAP + d + 1].d,
                                                         acnt + A_SNAP + d + 1);
        ++n;
      }
      kb_coarse_load<double, D><<<agrid(A_COARSE + d), blk, 0, s>>>(apt, LA[A_COARSE + d].d,
                                                                    acnt + A_COARSE + d, R);
      ++n;
    }
    const int gc = grid_for(b, L_COARSE + d);
    if (L[L_RESTR + d].cap > 0) {
      const int gr = grid_for(b, L_RESTR + d);
      if (b->mixed)
        kb_restrict<float, D><<<gr, blk, 0, s>>>(pt, L[L_RESTR + d].d, cnt + L_RESTR + d, R);
      else
        kb_restrict<double, D><<<gr, blk, 0, s>>>(pt, L[L_RESTR + d].d, cnt + L_RESTR + d, R);
      ++n;
    }
    if (b->mixed) {
      kb_coarse_load<float, D><<<gc, blk, 0, s>>>(pt, L[L_COARSE + d].d, cnt + L_COARSE + d,
                                                  R);
    } else {
      kb_coarse_load<double, D><<<gc, blk, 0, s>>>(pt, L[L_COARSE + d].d, cnt + L_COARSE + d,
                                                   R);
    }
    ++n;
  }
  {
    const int cap = std::max(1, L[L_TOPS].cap);
    const int gb = std::max(1, std::min(cap, 4 * b->nsm));
    kb_bottom<D><<<gb, BATCH_BOTTOM_THREADS, 0, s>>>(pt, L[L_TOPS].d, cnt + L_TOPS, nu);
    ++n;
    if (LA[A_TOPS].cap > 0) {
      const int ga = std::max(1, std::min(LA[A_TOPS].cap, 4 * b->nsm));
      kb_bottom<D><<<ga, BATCH_BOTTOM_THREADS, 0, s>>>(apt, LA[A_TOPS].d, acnt + A_TOPS, nu);
      ++n;
    }
  }
  for (int d = b->cap_depth - 1; d >= 0; --d) {
    if (D == 2) {
      // Records with fused stages are corrected by their post-smoothing stage.
      if (L[L_CORR + d].cap > 0) {
        const int gk = grid_for(b, L_CORR + d);
        if (b->mixed)
          kb_correct2<float><<<gk, blk, 0, s>>>(pt, L[L_CORR + d].d, cnt + L_CORR + d, R);
        else
          kb_correct2<double><<<gk, blk, 0, s>>>(pt, L[L_CORR + d].d, cnt + L_CORR + d, R);
      } else {
        --n;
      }
    } else {
      const int gf = grid_for(b, L_FINE + d);
      if (b->mixed)
        kb_correct<float, D><<<gf, blk, 0, s>>>(pt, L[L_FINE + d].d, cnt + L_FINE + d, R);
      else
        kb_correct<double, D><<<gf, blk, 0, s>>>(pt, L[L_FINE + d].d, cnt + L_FINE + d, R);
    }
    ++n;
    if (LA[A_FINE + d].cap > 0) {
      // CorrectFine and SetGhost(level, 0) (afas:513-515).
      kb_correct<double, D><<<agrid(A_FINE + d), blk, 0, s>>>(apt, LA[A_FINE + d].d,
                                                              acnt + A_FINE + d, R);
      ++n;
      aghost(d, 0);
    }
    relax(d, 1);
    arelax(d);
  }
  if (b->mixed) {
    kb_update<D><<<grid_for(b, L_UPD), blk, 0, s>>>(pt, L[L_UPD].d, cnt + L_UPD, R);
    launch_defect(0);
    n += 2;
  } else {
    kb_resid<D><<<gm, blk, 0, s>>>(pt, L[L_MASTER].d, cnt + L_MASTER, b->d_partials, R);
    ++n;
  }
  if (LA[A_MASTER].cap > 0) {
    // FillDown(solution) after the V-cycle (afas:73), then ErrorAFAS on the
    // finest level of each refined hierarchy.
    for (int d = 0; d < b->cap_depth; ++d)
      if (LA[A_FILL + d].cap > 0) {
        kb_filldown<D><<<agrid(A_FILL + d), blk, 0, s>>>(apt, LA[A_FILL + d].d,
                                                         acnt + A_FILL + d, R);
        ++n;
        aghost(d + 1, 0);
      }
    kb_resid<D><<<agrid(A_MASTER), blk, 0, s>>>(apt, LA[A_MASTER].d, acnt + A_MASTER,
                                                b->d_apartials, R);
    ++n;
  }
  const int gctl = std::max(1, std::min(b->bp.max_slots, 2 * b->nsm));
  k_batch_control<<<gctl, BLOCK_THREADS, 0, s>>>(pt, apt, b->d_cfg, b->d_state, b->d_log,
                                                 BSAM_BATCH_MAX_STEPS, b->d_out, b->d_partials,
                                                 b->d_apartials, b->d_ctl, b->bp.max_slots);
  k_batch_cond<<<1, 1, 0, s>>>(b->d_ctl, handle, in_graph);
  n += 2;
  b->kernels_per_tick = n;
}

int capture(bsam_batch* b) {
  CU(cudaStreamSynchronize(b->stream));
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
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
    e = cudaStreamBeginCaptureToGraph(b->stream, body, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      const bool prof = b->profiling;
      b->profiling = false;  // no events inside the graph
      if (b->bp.ndims == 2) tick_t<2>(b, handle, 1);
      else tick_t<3>(b, handle, 1);
      b->profiling = prof;
      cudaGraph_t captured = nullptr;
      e = cudaStreamEndCapture(b->stream, &captured);
    }
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    b->exec = nullptr;
    cudaGetLastError();
    return fail(b, BSAM_ERR_CUDA, std::string("tick graph: ") + cudaGetErrorString(e));
  }
  b->need_capture = false;
  ++b->st.captures;
  return BSAM_OK;
}

// Uploads list growth, counts and slot configuration; re-captures the tick
// graph when capacities or depths changed.
int flush(bsam_batch* b) {
  {
    const int rc = amr_flush(b);
    if (rc) return rc;
  }
  for (int l = 0; l < NLIST; ++l) {
    List& L = b->lists[l];
    const int n = (int)L.h.size();
    if (n > L.cap) {
      CU(cudaStreamSynchronize(b->stream));
      if (L.d) cudaFree(L.d);
      L.d = nullptr;
      int cap = std::max(256, L.cap);
      while (cap < n) cap *= 2;
      if (cudaMalloc(&L.d, sizeof(Item) * cap) != cudaSuccess) {
        L.cap = 0;
        return fail(b, BSAM_ERR_NOMEM, "work list allocation failed");
      }
      L.cap = cap;
      L.uploaded = 0;
      b->need_capture = true;
      if (l == L_MASTER && cap > b->partials_cap) {
        if (b->d_partials) cudaFree(b->d_partials);
        b->d_partials = nullptr;
        if (cudaMalloc(&b->d_partials, sizeof(double) * cap) != cudaSuccess)
          return fail(b, BSAM_ERR_NOMEM, "partials allocation failed");
        b->partials_cap = cap;
      }
    }
    if (L.uploaded < n) {
      const int rc = stage_copy(b, L.d + L.uploaded, L.h.data() + L.uploaded,
                                sizeof(Item) * (n - L.uploaded));
      if (rc) return rc;
      L.uploaded = n;
    }
  }
  std::vector<int> counts(NLIST);
  for (int l = 0; l < NLIST; ++l) counts[l] = (int)b->lists[l].h.size();
  if (counts != b->counts_dev) {
    const int rc = stage_copy(b, b->d_counts, counts.data(), sizeof(int) * NLIST);
    if (rc) return rc;
    b->counts_dev = counts;
  }
  if (b->cfg_dirty) {
    const int rc = stage_copy(b, b->d_cfg, b->h_cfg.data(), sizeof(SlotCfg) * b->h_cfg.size());
    if (rc) return rc;
    b->cfg_dirty = false;
  }
  int depth = 1;
  for (auto& S : b->slots)
    if (S.used) depth = std::max(depth, S.ntop);
  if (depth > b->cap_depth) {
    b->cap_depth = depth;
    b->need_capture = true;
  }
  stage_commit(b);
  if (b->need_capture) return capture(b);
  return BSAM_OK;
}

// Regrids every refined hierarchy waiting between two time steps (phase
// SLOT_REGRID as the completed work shows it; its records are inactive, so
// no queued tick touches its fields) and starts its next step: the native
// driver's AMR(rootlevel) and the start of MultigridIterations on the
// problem's own engine and stream, then its new records and tiles, which
// the batch's stream takes only after an event of the engine's.  The
// regrids touch only their own engines and run on host threads side by
// side (their host clustering and device work overlap); the batch's tables
// are then updated on this thread.
int amr_service(bsam_batch* b) {
  std::vector<int> due;
  for (size_t i = 0; i < b->slots.size(); ++i) {
    const SlotPlan& S = b->slots[i];
    if (S.used && S.amr && ((volatile SlotOut*)b->h_out)[i].phase == SLOT_REGRID)
      due.push_back((int)i);
  }
  if (due.empty()) return BSAM_OK;
  const auto t_start = std::chrono::steady_clock::now();
  std::vector<int> rcs(due.size(), BSAM_OK);
  std::vector<std::string> why(due.size());
  std::atomic<size_t> next{0};
  auto work = [&]() {
    cudaSetDevice(b->device);
    for (size_t k; (k = next.fetch_add(1)) < due.size();) {
      SlotPlan& S = b->slots[due[k]];
      int rc = bsam_amr_regrid(S.drv);
      if (rc == BSAM_OK) rc = engine_prologue(S.eng);
      if (rc == BSAM_OK) rc = engine_view(S.eng, S.view);
      if (rc == BSAM_OK && cudaEventRecord(S.ready, engine_stream(S.eng)) != cudaSuccess)
        rc = BSAM_ERR_CUDA;
      if (rc != BSAM_OK) why[k] = bsam_gpu_last_error(S.eng);
      rcs[k] = rc;
    }
  };
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  // Default: the host's hardware threads, at most 16 (measured on 16 cores,
  // 32 problems of the sustained AMR workload: 16 threads 1,926-1,951
  // time-steps/s, 8 threads 1,754-1,830, 4 threads 1,566).
  const int want = b->tuning.regrid_threads > 0 ? b->tuning.regrid_threads
                                                : (int)std::min(16u, hw);
  const int nt = (int)std::min<size_t>(due.size(), (size_t)want);
  if (nt <= 1) {
    work();
  } else {
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
  }
  b->st.regrids += (int64_t)due.size();
  b->st.regrid_s +=
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  // A problem whose regrid (or new hierarchy) fails ends as SLOT_FAILED
  // (its driver's state is not that of a completed regrid); the others start
  // their next step; the first failure is returned.
  int first_rc = BSAM_OK;
  std::string first_why;
  for (size_t k = 0; k < due.size(); ++k) {
    const int i = due[k];
    SlotPlan& S = b->slots[i];
    volatile SlotOut* o = b->h_out + i;
    const int step = o->step, vcycles = o->vcycles;
    int rc = rcs[k];
    if (rc == BSAM_OK) rc = amr_plan(b, S);
    if (rc != BSAM_OK) {
      if (first_rc == BSAM_OK) {
        first_rc = rc;
        first_why = why[k].empty() ? b->err : why[k];
      }
      SlotState st{SLOT_FAILED, step, 0, vcycles};
      const int src = stage_copy(b, b->d_state + i, &st, sizeof(st));
      if (src) return src;
      o->phase = SLOT_FAILED;
      continue;
    }
    CU(cudaStreamWaitEvent(b->stream, S.ready, 0));
    if ((int)b->h_apt.size() > 2 * live_amr_records(b) + 4096) {
      rc = amr_compact(b);
      if (rc) return rc;
    }
    amr_append(b, i, true);
    SlotState st{SLOT_RUNNING, step, 0, vcycles};
    rc = stage_copy(b, b->d_state + i, &st, sizeof(st));
    if (rc) return rc;
    o->phase = SLOT_RUNNING;
  }
  if (first_rc != BSAM_OK)
    return fail(b, first_rc, "regrid of a refined problem: " + first_why);
  return BSAM_OK;
}

bool amr_waiting(bsam_batch* b) {
  for (size_t i = 0; i < b->slots.size(); ++i)
    if (b->slots[i].used && b->slots[i].amr &&
        ((volatile SlotOut*)b->h_out)[i].phase == SLOT_REGRID)
      return true;
  return false;
}

}  // namespace

extern "C" {

const char* bsam_batch_last_error(bsam_batch* b) { return b ? b->err.c_str() : "null handle"; }

int bsam_batch_create(bsam_batch** out, int device, const bsam_batch_params* p) {
  if (!out || !p) return BSAM_ERR_ARG;
  *out = nullptr;
  if (p->ndims < 2 || p->ndims > 3 || p->nsmoothingpasses < 1 || p->maxvcycles < 1 ||
      p->max_slots < 1 || p->max_slots > (1 << 20) / RMAX || p->pool_bytes < 0 ||
      p->bottom_cells < 0 || p->bottom_cells > BOTTOM_MAX_CELLS)
    return BSAM_ERR_ARG;
  if (p->precision != BSAM_PREC_FP64 && p->precision != BSAM_PREC_MIXED)
    return BSAM_ERR_UNSUPPORTED;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return BSAM_ERR_NODEVICE;
  if (cudaSetDevice(device) != cudaSuccess) return BSAM_ERR_NODEVICE;
  bsam_batch* b = new bsam_batch();
  b->device = device;
  b->bp = *p;
  if (b->bp.bottom_cells == 0) b->bp.bottom_cells = DEFAULT_BOTTOM_CELLS;
  b->mixed = p->precision == BSAM_PREC_MIXED;
  cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, device);
  const int ns = p->max_slots;
  size_t pool = (size_t)p->pool_bytes;
  if (pool == 0) {
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    pool = fr / 2;
  }
  pool = (size_t)roundup((int64_t)pool, 4096);
  bool ok = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&b->xstream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->xin_ready, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->xin_free, cudaEventDisableTiming) == cudaSuccess &&
            cudaMalloc(&b->d_pool, pool) == cudaSuccess &&
            cudaMalloc(&b->d_pt, sizeof(DevPatch) * ns * RMAX) == cudaSuccess &&
            cudaMalloc(&b->d_tmaps, sizeof(CUtensorMap) * NMAPS * ns * RMAX) == cudaSuccess &&
            cudaMalloc(&b->d_cfg, sizeof(SlotCfg) * ns) == cudaSuccess &&
            cudaMalloc(&b->d_state, sizeof(SlotState) * ns) == cudaSuccess &&
            cudaMalloc(&b->d_log, sizeof(StepLog) * ns * BSAM_BATCH_MAX_STEPS) == cudaSuccess &&
            cudaHostAlloc(&b->h_out, sizeof(SlotOut) * ns, cudaHostAllocMapped) == cudaSuccess &&
            cudaMalloc(&b->d_ctl, sizeof(BatchCtl)) == cudaSuccess &&
            cudaMalloc(&b->d_status, sizeof(DevStatus)) == cudaSuccess &&
            cudaMallocHost(&b->h_status, sizeof(DevStatus)) == cudaSuccess &&
            cudaMalloc(&b->d_counts, sizeof(int) * NLIST) == cudaSuccess &&
            cudaMalloc(&b->d_acounts, sizeof(int) * ANLIST) == cudaSuccess;
  if (ok) ok = cudaHostGetDevicePointer((void**)&b->d_out, b->h_out, 0) == cudaSuccess;
  if (ok)
    ok = cudaFuncSetAttribute(kb_smooth2<float, true, 3>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)Fused2<float>::SMEM) == cudaSuccess &&
         cudaFuncSetAttribute(kb_smooth2<float, true, 4>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)Fused2<float>::SMEM) == cudaSuccess &&
         cudaFuncSetAttribute(kb_smooth2<double, false, 3>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)Fused2<double>::SMEM) == cudaSuccess &&
         cudaFuncSetAttribute(kb_smooth2<double, false, 4>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)Fused2<double>::SMEM) == cudaSuccess &&
         cudaFuncSetAttribute(kb_smooth2<float, true, 2, 2>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(2 * Fused2<float>::smem(true))) == cudaSuccess &&
         cudaFuncSetAttribute(kb_smooth2<double, false, 2, 2>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(2 * Fused2<double>::smem(false))) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    bsam_batch_destroy(b);
    return BSAM_ERR_NOMEM;
  }
  b->pool_bytes = pool;
  b->free_[0] = pool;
  b->slots.assign(ns, SlotPlan{});
  b->h_cfg.assign(ns, SlotCfg{});
  std::memset(b->h_out, 0, sizeof(SlotOut) * ns);
  cudaMemsetAsync(b->d_pt, 0, sizeof(DevPatch) * ns * RMAX, b->stream);  // active = 0
  cudaMemsetAsync(b->d_cfg, 0, sizeof(SlotCfg) * ns, b->stream);
  cudaMemsetAsync(b->d_state, 0, sizeof(SlotState) * ns, b->stream);  // SLOT_IDLE
  cudaMemsetAsync(b->d_ctl, 0, sizeof(BatchCtl), b->stream);
  cudaMemsetAsync(b->d_counts, 0, sizeof(int) * NLIST, b->stream);
  cudaMemsetAsync(b->d_acounts, 0, sizeof(int) * ANLIST, b->stream);
  cudaMemsetAsync(b->d_status, 0, sizeof(DevStatus), b->stream);
  b->counts_dev.assign(NLIST, 0);
  b->acounts_dev.assign(ANLIST, 0);
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) {
    bsam_batch_destroy(b);
    return BSAM_ERR_CUDA;
  }
  *out = b;
  return BSAM_OK;
}

int bsam_batch_destroy(bsam_batch* b) {
  if (!b) return BSAM_ERR_ARG;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  for (auto& e : b->ev_pool) {
    cudaEventDestroy(e.first);
    cudaEventDestroy(e.second);
  }
  for (auto& L : b->lists)
    if (L.d) cudaFree(L.d);
  for (auto& L : b->alists)
    if (L.d) cudaFree(L.d);
  for (auto& S : b->slots)
    if (S.ready) cudaEventDestroy(S.ready);
  if (b->d_apt) cudaFree(b->d_apt);
  if (b->d_aovl) cudaFree(b->d_aovl);
  if (b->d_acounts) cudaFree(b->d_acounts);
  if (b->d_apartials) cudaFree(b->d_apartials);
  for (auto& c : b->chunks)
    if (c.ev) b->free_events.push_back(c.ev);
  std::sort(b->free_events.begin(), b->free_events.end());
  b->free_events.erase(std::unique(b->free_events.begin(), b->free_events.end()),
                       b->free_events.end());
  for (auto e : b->free_events) cudaEventDestroy(e);
  if (b->stage) cudaFreeHost(b->stage);
  if (b->xstream) cudaStreamSynchronize(b->xstream);
  if (b->d_xin) cudaFree(b->d_xin);
  if (b->d_xout) cudaFree(b->d_xout);
  if (b->xin_ready) cudaEventDestroy(b->xin_ready);
  if (b->xin_free) cudaEventDestroy(b->xin_free);
  if (b->xstream) cudaStreamDestroy(b->xstream);
  if (b->d_partials) cudaFree(b->d_partials);
  if (b->d_counts) cudaFree(b->d_counts);
  if (b->h_status) cudaFreeHost(b->h_status);
  if (b->d_status) cudaFree(b->d_status);
  if (b->d_ctl) cudaFree(b->d_ctl);
  if (b->h_out) cudaFreeHost(b->h_out);
  if (b->d_log) cudaFree(b->d_log);
  if (b->d_state) cudaFree(b->d_state);
  if (b->d_cfg) cudaFree(b->d_cfg);
  if (b->d_pt) cudaFree(b->d_pt);
  if (b->d_tmaps) cudaFree(b->d_tmaps);
  if (b->d_pool) cudaFree(b->d_pool);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return BSAM_OK;
}

int bsam_batch_set_tuning(bsam_batch* b, const bsam_batch_tuning* t) {
  if (!b || !t || t->grid_ctas < 0 || t->eager < 0 || t->eager > 1 || t->per_pass < 0 ||
      t->per_pass > 1 || t->fused_ctas < 0 ||
      (t->fused_occ != 0 && (t->fused_occ < 2 || t->fused_occ > 4)) || t->tile_chunk < 0 ||
      t->tile_chunk > 64 || t->fused_chunk < 0 || t->fused_chunk > 64 || t->regrid_threads < 0 ||
      t->regrid_threads > 64)
    return BSAM_ERR_ARG;
  b->tuning = *t;
  b->need_capture = true;
  return BSAM_OK;
}

int bsam_batch_footprint(bsam_batch* b, const bsam_batch_problem* prob, int64_t* bytes) {
  if (!b || !prob || !bytes) return BSAM_ERR_ARG;
  SlotPlan S;
  const int rc = plan_slot(b, prob, 0, nullptr, S);
  if (rc) return rc;
  *bytes = (int64_t)S.bytes;
  return BSAM_OK;
}

// Admission of one problem; its initial state is either copied from the host
// (q0) or drawn on the device (init).
struct SeedInit {
  uint64_t seed;
  double cbar, amp;
};

// Host side of one admission: a free slot (compacting the lists if only
// retired slots are left), a pool region and the slot's records.
static int reserve(bsam_batch* b, const bsam_batch_problem* prob, int* slot) {
  SlotPlan probe;
  int rc = plan_slot(b, prob, 0, nullptr, probe);
  if (rc) return rc;
  // A free slot whose old tiles are gone from the lists; compact if only
  // retired ones are left.
  int s = -1;
  bool any_stale = false;
  for (size_t i = 0; i < b->slots.size(); ++i) {
    if (b->slots[i].used) continue;
    if (!b->slots[i].stale) {
      s = (int)i;
      break;
    }
    any_stale = true;
  }
  if (s < 0 && !any_stale) return fail(b, BSAM_ERR_NOMEM, "no free slot");
  size_t off = 0;
  if (!pool_alloc(b, probe.bytes, &off)) return fail(b, BSAM_ERR_NOMEM, "pool is full");
  if (s < 0) {
    compact(b);
    for (size_t i = 0; i < b->slots.size(); ++i)
      if (!b->slots[i].used) {
        s = (int)i;
        break;
      }
  }
  SlotPlan& S = b->slots[s];
  const int rec0 = s * RMAX;
  rc = plan_slot(b, prob, rec0, b->d_pool + off, S);
  if (rc) {
    pool_free(b, off, probe.bytes);
    return rc;
  }
  S.used = true;
  S.stale = false;
  S.off = off;
  S.amr = false;
  S.drv = nullptr;
  S.eng = nullptr;
  *slot = s;
  return BSAM_OK;
}

// Host bookkeeping of an admitted slot, once its device work is queued.
static void enlist(bsam_batch* b, int s, const bsam_batch_problem* prob) {
  const SlotPlan& S = b->slots[s];
  const int rec0 = s * RMAX;
  SlotCfg& C = b->h_cfg[s];
  C.kind = SLOT_UNIFORM;
  C.rec0 = rec0;
  C.nrec = S.nrec;
  C.master = rec0 + S.master;
  C.nsteps = prob->nsteps;
  C.maxv = b->bp.maxvcycles;
  C.denom = 2.0 * (double)S.cells;
  C.tol = b->bp.qerrortol;
  append_items(b, s);
  volatile SlotOut* o = b->h_out + s;
  o->step = 0;
  o->vcycles = 0;
  o->phase = SLOT_RUNNING;
}

static double seed_k2(const bsam_batch_problem* prob, const DevPatch& M) {
  return (prob->eps * prob->eps) / (M.h * M.h);
}

static int admit(bsam_batch* b, const bsam_batch_problem* prob, const double* q0,
                 const SeedInit* init, int* slot) {
  if (!b || !prob || (!q0 && !init) || !slot) return BSAM_ERR_ARG;
  CU(cudaSetDevice(b->device));
  int s = -1;
  int rc = reserve(b, prob, &s);
  if (rc) return rc;
  SlotPlan& S = b->slots[s];
  const int rec0 = s * RMAX;
  const size_t off = S.off;
  const int nd = b->bp.ndims;
  // Fresh fields, records, the initial state and its ghosts.
  CU(cudaMemsetAsync(b->d_pool + off, 0, S.bytes, b->stream));
  rc = stage_copy(b, b->d_pt + rec0, S.recs.data(), sizeof(DevPatch) * S.nrec);
  if (rc) return rc;
  for (int r = 0; r < S.nrec; ++r)
    if (S.recs[r].tmaps) {
      rc = stage_copy(b, b->d_tmaps + (size_t)(rec0 + r) * NMAPS, &S.maps[(size_t)r * NMAPS],
                      sizeof(CUtensorMap) * NMAPS);
      if (rc) return rc;
    }
  const DevPatch& M = S.recs[S.master];
  const int e0 = M.n[0] + 2, e1 = M.n[1] + 2, e2 = nd == 3 ? M.n[2] + 2 : 1;
  const size_t hcomp = (size_t)e0 * e1 * e2;
  if (q0) {
    char* st = stage_alloc(b, sizeof(double) * 2 * hcomp);
    if (!st) return fail(b, BSAM_ERR_NOMEM, "pinned staging allocation failed");
    std::memcpy(st, q0, sizeof(double) * 2 * hcomp);
    for (int c = 0; c < 2; ++c)
      CU(cudaMemcpy2DAsync(M.q[c], M.sy * sizeof(double), st + c * hcomp * sizeof(double),
                           e0 * sizeof(double), e0 * sizeof(double), (size_t)e1 * e2,
                           cudaMemcpyHostToDevice, b->stream));
  } else {
    const double k2 = seed_k2(prob, M);
    const int64_t ncell = S.cells;
    const int gi = (int)std::min<int64_t>((ncell + 255) / 256, 16 * b->nsm);
    if (nd == 2)
      k_init_seeded<2><<<gi, 256, 0, b->stream>>>(b->d_pt, rec0 + S.master, init->seed,
                                                   init->cbar, init->amp, k2);
    else
      k_init_seeded<3><<<gi, 256, 0, b->stream>>>(b->d_pt, rec0 + S.master, init->seed,
                                                   init->cbar, init->amp, k2);
  }
  const int64_t total = (int64_t)hcomp;
  const int nb = (int)((total + 255) / 256);
  if (nd == 2) k_setbc<double, 2><<<nb, 256, 0, b->stream>>>(b->d_pt, rec0 + S.master, total);
  else k_setbc<double, 3><<<nb, 256, 0, b->stream>>>(b->d_pt, rec0 + S.master, total);
  CU(cudaGetLastError());
  SlotState z{SLOT_RUNNING, 0, 0, 0};
  rc = stage_copy(b, b->d_state + s, &z, sizeof(SlotState));
  if (rc) return rc;
  enlist(b, s, prob);
  stage_commit(b);
  *slot = s;
  return BSAM_OK;
}

// Many admissions with their device work batched: one launch zeroes the
// admitted pool regions, one scatters every record, tensor map and slot
// state from page-locked staging, one draws the seeded states (or one pitched
// copy per component and problem from q0s), one sets their ghosts.
static int admit_many(bsam_batch* b, int n, const bsam_batch_problem* probs,
                      const double* const* q0s, const SeedInit* inits, int* slots) {
  if (!b || n < 0 || (n > 0 && (!probs || !slots)) || (!q0s && !inits)) return BSAM_ERR_ARG;
  if (n == 0) return 0;
  CU(cudaSetDevice(b->device));
  // Every problem is checked before any is admitted, and the transfer
  // buffer is sized for all of them before any slot is taken.
  size_t xwords = 0;
  for (int k = 0; k < n; ++k) {
    SlotPlan probe;
    const int rc = plan_slot(b, &probs[k], 0, nullptr, probe);
    if (rc) return rc;
    if (q0s && !q0s[k]) return fail(b, BSAM_ERR_ARG, "a q0 pointer is NULL");
    const DevPatch& M = probe.recs[probe.master];
    xwords += 2 * (size_t)(M.n[0] + 2) * (M.n[1] + 2) * (b->bp.ndims == 3 ? M.n[2] + 2 : 1);
  }
  double* xfer = nullptr;
  if (q0s && !(xfer = xfer_reserve(b, &b->d_xin, &b->xin_words, xwords)))
    return fail(b, BSAM_ERR_NOMEM, "transfer buffer allocation failed");
  std::vector<int> adm;
  for (int k = 0; k < n; ++k) slots[k] = -1;
  // Admission stops at the first problem that does not fit: the admitted
  // ones are problems 0 .. na-1.  Each is listed at once, so that a
  // compaction by a later reservation keeps its tiles exactly once.
  for (int k = 0; k < n; ++k) {
    int s = -1;
    const int rc = reserve(b, &probs[k], &s);
    if (rc == BSAM_ERR_NOMEM) break;
    if (rc) return rc;
    enlist(b, s, &probs[k]);
    adm.push_back(s);
    slots[k] = s;
  }
  const int na = (int)adm.size();
  if (na == 0) return 0;
  const int nd = b->bp.ndims;
  // Staging layout: spans, zero spans, seed tasks, master records, then the
  // words the spans copy (records, tensor maps, slot states).
  int nspan = 0;
  size_t words = 0;
  for (int s : adm) {
    const SlotPlan& S = b->slots[s];
    nspan += 2;  // records, slot state
    words += (sizeof(DevPatch) * S.nrec + sizeof(SlotState) + 7) / 8 + 1;
    for (int r = 0; r < S.nrec; ++r)
      if (S.recs[r].tmaps) {
        ++nspan;
        words += sizeof(CUtensorMap) * NMAPS / 8;
      }
  }
  static_assert(sizeof(DevPatch) % 8 == 0 && sizeof(SlotState) % 8 == 0 &&
                    sizeof(CUtensorMap) % 8 == 0,
                "staged records are copied as 8-byte words");
  // Packed root states of the q0s in the device transfer buffer.
  std::vector<size_t> xo((size_t)na + 1, 0);
  for (int a = 0; a < na; ++a) {
    const DevPatch& M = b->slots[adm[a]].recs[b->slots[adm[a]].master];
    xo[a + 1] = xo[a] + 2 * (size_t)(M.n[0] + 2) * (M.n[1] + 2) * (nd == 3 ? M.n[2] + 2 : 1);
  }
  const size_t bytes = sizeof(RowsTask) * na + sizeof(WordSpan) * nspan +
                       sizeof(ZeroSpan) * na + sizeof(SeedTask) * na + sizeof(int) * (na + 1) +
                       8 * words + 64;
  char* st = stage_alloc(b, bytes);
  if (!st) return fail(b, BSAM_ERR_NOMEM, "pinned staging allocation failed");
  RowsTask* rows = reinterpret_cast<RowsTask*>(st);
  WordSpan* spans = reinterpret_cast<WordSpan*>(rows + na);
  ZeroSpan* zs = reinterpret_cast<ZeroSpan*>(spans + nspan);
  SeedTask* tasks = reinterpret_cast<SeedTask*>(zs + na);
  int* masters = reinterpret_cast<int*>(tasks + na);
  uint64_t* w = reinterpret_cast<uint64_t*>(
      (reinterpret_cast<uintptr_t>(masters + na) + 7) & ~uintptr_t(7));
  int sp = 0;
  int64_t maxz = 0, maxw = 0, maxc = 0;
  for (int a = 0; a < na; ++a) {
    const int s = adm[a];
    const SlotPlan& S = b->slots[s];
    const int rec0 = s * RMAX;
    const DevPatch& M = S.recs[S.master];
    zs[a] = ZeroSpan{reinterpret_cast<uint64_t*>(b->d_pool + S.off), (int64_t)(S.bytes / 8)};
    maxz = std::max<int64_t>(maxz, zs[a].n);
    masters[a] = rec0 + S.master;
    if (inits)
      tasks[a] = SeedTask{rec0 + S.master, 0, inits[a].seed, inits[a].cbar, inits[a].amp,
                          seed_k2(&probs[a], M)};
    maxc = std::max<int64_t>(maxc, S.cells);
    auto add = [&](void* dst, const void* src, size_t nbytes) {
      std::memcpy(w, src, nbytes);
      spans[sp++] = WordSpan{w, static_cast<uint64_t*>(dst), (int64_t)(nbytes / 8)};
      maxw = std::max<int64_t>(maxw, (int64_t)(nbytes / 8));
      w += nbytes / 8;
    };
    add(b->d_pt + rec0, S.recs.data(), sizeof(DevPatch) * S.nrec);
    for (int r = 0; r < S.nrec; ++r)
      if (S.recs[r].tmaps)
        add(b->d_tmaps + (size_t)(rec0 + r) * NMAPS, &S.maps[(size_t)r * NMAPS],
            sizeof(CUtensorMap) * NMAPS);
    const SlotState z{SLOT_RUNNING, 0, 0, 0};
    add(b->d_state + s, &z, sizeof(SlotState));
  }
  auto gx = [&](int64_t m) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((m + 255) / 256, 64)); };
  k_zero_spans<<<dim3(gx(maxz), na), 256, 0, b->stream>>>(zs);
  k_word_spans<<<dim3(gx(maxw), sp), 256, 0, b->stream>>>(spans);
  if (inits) {
    if (nd == 2) k_init_seeded_list<2><<<dim3(gx(maxc), na), 256, 0, b->stream>>>(b->d_pt, tasks);
    else k_init_seeded_list<3><<<dim3(gx(maxc), na), 256, 0, b->stream>>>(b->d_pt, tasks);
  } else {
    // q0s: one contiguous copy per problem into the transfer buffer, on the
    // copy stream (read asynchronously from page-locked memory, alongside
    // the ticks already queued), then one launch on the engine's stream
    // spreads the rows into the pitched fields.
    CU(cudaStreamWaitEvent(b->xstream, b->xin_free, 0));
    int64_t maxr = 0;
    for (int a = 0; a < na; ++a) {
      const SlotPlan& S = b->slots[adm[a]];
      const DevPatch& M = S.recs[S.master];
      const int e0 = M.n[0] + 2;
      const int64_t nrow = (int64_t)(M.n[1] + 2) * (nd == 3 ? M.n[2] + 2 : 1);
      rows[a] = RowsTask{xfer + xo[a], {static_cast<double*>(M.q[0]), static_cast<double*>(M.q[1])},
                         nrow, M.sy, e0, 0};
      maxr = std::max(maxr, 2 * nrow);
      CU(cudaMemcpyAsync(xfer + xo[a], q0s[a], sizeof(double) * (xo[a + 1] - xo[a]),
                         cudaMemcpyHostToDevice, b->xstream));
    }
    CU(cudaEventRecord(b->xin_ready, b->xstream));
    CU(cudaStreamWaitEvent(b->stream, b->xin_ready, 0));
    const unsigned gr = (unsigned)std::max<int64_t>(1, std::min<int64_t>((maxr + 7) / 8, 64));
    k_rows_list<true><<<dim3(gr, na), 256, 0, b->stream>>>(rows);
    CU(cudaEventRecord(b->xin_free, b->stream));
  }
  if (nd == 2) k_setbc_list<double, 2><<<dim3(gx(maxc), na), 256, 0, b->stream>>>(b->d_pt, masters);
  else k_setbc_list<double, 3><<<dim3(gx(maxc), na), 256, 0, b->stream>>>(b->d_pt, masters);
  CU(cudaGetLastError());
  stage_commit(b);
  return na;
}

int bsam_batch_submit(bsam_batch* b, const bsam_batch_problem* prob, const double* q0,
                      int* slot) {
  if (!q0) return BSAM_ERR_ARG;
  return admit(b, prob, q0, nullptr, slot);
}

int bsam_batch_submit_seeded(bsam_batch* b, const bsam_batch_problem* prob, uint64_t seed,
                             double cbar, double amp, int* slot) {
  const SeedInit init{seed, cbar, amp};
  return admit(b, prob, nullptr, &init, slot);
}

int bsam_batch_submit_many(bsam_batch* b, int n, const bsam_batch_problem* probs,
                           const double* const* q0s, int* slots) {
  if (!q0s) return BSAM_ERR_ARG;
  return admit_many(b, n, probs, q0s, nullptr, slots);
}

int bsam_batch_submit_seeded_many(bsam_batch* b, int n, const bsam_batch_problem* probs,
                                  const uint64_t* seeds, const double* cbar, const double* amp,
                                  int* slots) {
  if (n > 0 && (!seeds || !cbar || !amp)) return BSAM_ERR_ARG;
  std::vector<SeedInit> init((size_t)std::max(n, 0));
  for (int k = 0; k < n; ++k) init[k] = SeedInit{seeds[k], cbar[k], amp[k]};
  return admit_many(b, n, probs, nullptr, init.data(), slots);
}

int bsam_batch_submit_amr(bsam_batch* b, bsam_amr* a, int nsteps, int* slot) {
  if (!b || !a || !slot || nsteps < 1 || nsteps > BSAM_BATCH_MAX_STEPS) return BSAM_ERR_ARG;
  CU(cudaSetDevice(b->device));
  bsam_gpu* h = amr_engine(a);
  if (engine_device(h) != b->device)
    return fail(b, BSAM_ERR_ARG, "the driver's engine is on another device");
  for (const auto& S : b->slots)
    if (S.used && S.amr && S.drv == a) return fail(b, BSAM_ERR_STATE, "driver already in the batch");
  {
    // The hierarchy as it stands must fit the batch (checked again after
    // every regrid).
    SlotPlan probe;
    int rc = engine_view(h, probe.view);
    if (rc) return fail(b, rc, "the driver's engine holds no hierarchy");
    rc = amr_plan(b, probe);
    if (rc) return rc;
  }
  int s = -1;
  bool any_stale = false;
  for (size_t i = 0; i < b->slots.size(); ++i) {
    if (b->slots[i].used) continue;
    if (!b->slots[i].stale) {
      s = (int)i;
      break;
    }
    any_stale = true;
  }
  if (s < 0 && !any_stale) return fail(b, BSAM_ERR_NOMEM, "no free slot");
  if (s < 0) {
    compact(b);
    for (size_t i = 0; i < b->slots.size(); ++i)
      if (!b->slots[i].used) {
        s = (int)i;
        break;
      }
  }
  SlotPlan& S = b->slots[s];
  S = SlotPlan{};
  S.used = true;
  S.amr = true;
  S.drv = a;
  S.eng = h;
  S.nsteps = nsteps;
  S.prob.nsteps = nsteps;
  CU(cudaEventCreateWithFlags(&S.ready, cudaEventDisableTiming));
  SlotCfg& C = b->h_cfg[s];
  C = SlotCfg{};
  C.kind = SLOT_AMR;
  C.nsteps = nsteps;
  b->cfg_dirty = true;
  // Waits between two time steps from the start: the first step's regrid
  // runs at the next advance.
  SlotState st{SLOT_REGRID, 0, 0, 0};
  const int rc = stage_copy(b, b->d_state + s, &st, sizeof(st));
  if (rc) return rc;
  volatile SlotOut* o = b->h_out + s;
  o->step = 0;
  o->vcycles = 0;
  o->phase = SLOT_REGRID;
  *slot = s;
  return BSAM_OK;
}

int bsam_batch_busy(bsam_batch* b) {
  if (!b) return BSAM_ERR_ARG;
  cudaSetDevice(b->device);
  const cudaError_t e = cudaStreamQuery(b->stream);
  if (e == cudaSuccess) return 0;
  if (e == cudaErrorNotReady) return 1;
  return fail(b, BSAM_ERR_CUDA, std::string("stream query: ") + cudaGetErrorString(e));
}

int bsam_batch_advance(bsam_batch* b, int max_ticks) {
  if (!b || max_ticks < 1) return BSAM_ERR_ARG;
  CU(cudaSetDevice(b->device));
  int rc = amr_service(b);
  if (rc) return rc;
  rc = flush(b);
  if (rc) return rc;
  k_batch_budget<<<1, 1, 0, b->stream>>>(b->d_ctl, max_ticks);
  CU(cudaGetLastError());
  if (!b->tuning.eager && !b->profiling) {
    CU(cudaGraphLaunch(b->exec, b->stream));
    return BSAM_OK;
  }
  // Eager ticks: exactly max_ticks; with profiling, one tick at a time so
  // that each timed stage is attributed to the problems running in it.
  const cudaGraphConditionalHandle none = 0;
  for (int t = 0; t < max_ticks; ++t) {
    // Algorithmic bytes of the finest-depth stages of the problems running
    // in this tick, per cell of their finest working level (s = bytes per
    // value of that level, sp = of its parent):
    //  pre-smoothing: read f1, f2 (+ the base, correction form) and, unless
    //    the correction starts from zero, the state; write the smoothed
    //    state; restrict into the parent (its q and qs, + base): 2 s + 1 s
    //    (base) + 0 / 2 s (state) + 2 s + (4 | 5) sp / 4;
    //  post-smoothing: read the pre-smoothed state, f1, f2 (+ base) and the
    //    parent's q and qs for the correction (4 sp / 4); write the state,
    //    or, with the FP64 update, read and write the FP64 master (32).
    double pre_bytes = 0.0, post_bytes = 0.0;
    if (b->profiling) {
      CU(cudaStreamSynchronize(b->stream));
      const bool fused = b->bp.ndims == 2 && !b->tuning.per_pass;
      for (size_t s = 0; s < b->slots.size(); ++s) {
        const SlotPlan& S = b->slots[s];
        if (!S.used || ((volatile SlotOut*)b->h_out)[s].phase != SLOT_RUNNING || S.ntop < 1)
          continue;
        const int first = b->mixed ? 1 : 0;  // record of depth 0
        const DevPatch& W = S.recs[first];
        const double sw = W.prec == PREC_F32 ? 4.0 : 8.0;
        const double sp = S.recs[first + 1].prec == PREC_F32 ? 4.0 : 8.0;
        const double cells = (double)S.cells;
        if (fused) {
          const bool delta = W.delta != 0;
          pre_bytes += cells * (2 * sw + (delta ? sw : 0.0) + (delta ? 0.0 : 2 * sw) + 2 * sw +
                                (delta ? 5.0 : 4.0) * sp / 4.0);
          post_bytes += cells * (4 * sw + (delta ? sw : 0.0) + sp +
                                 (b->mixed ? 32.0 : 2 * sw));
        } else {
          // One launch per colour pass: each pass reads and writes the state
          // and reads f (and the base): counted once per stage as 6 s.
          pre_bytes += cells * 6 * sw;
          post_bytes += cells * 6 * sw;
        }
      }
    }
    b->ev_used = 0;
    if (b->bp.ndims == 2) tick_t<2>(b, none, 0);
    else tick_t<3>(b, none, 0);
    CU(cudaGetLastError());
    if (b->profiling) {
      CU(cudaStreamSynchronize(b->stream));
      for (size_t e = 0; e < b->ev_used; ++e) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, b->ev_pool[e].first, b->ev_pool[e].second) == cudaSuccess) {
          b->st.smooth_ms += ms;
          b->st.smooth_stages += 1;
          b->st.smooth_bytes += b->ev_post[e] ? post_bytes : pre_bytes;
        }
      }
      b->ev_used = 0;
    }
  }
  return BSAM_OK;
}

int bsam_batch_profile(bsam_batch* b, int enable) {
  if (!b) return BSAM_ERR_ARG;
  if (enable) {
    b->st.smooth_ms = 0.0;
    b->st.smooth_stages = 0;
    b->st.smooth_bytes = 0.0;
  }
  b->profiling = enable != 0;
  return BSAM_OK;
}

int bsam_batch_sync(bsam_batch* b) {
  if (!b) return BSAM_ERR_ARG;
  CU(cudaSetDevice(b->device));
  CU(cudaStreamSynchronize(b->stream));
  int32_t kerr = 0;
  CU(cudaMemcpy(&kerr, &b->d_ctl->kerr, sizeof(kerr), cudaMemcpyDeviceToHost));
  if (kerr) return fail(b, BSAM_ERR_CUDA, "a fused smoothing stage timed out waiting for its copies");
  return BSAM_OK;
}

static int running_slots(bsam_batch* b) {
  int n = 0;
  for (size_t s = 0; s < b->slots.size(); ++s)
    if (b->slots[s].used && ((volatile SlotOut*)b->h_out)[s].phase == SLOT_RUNNING) ++n;
  return n;
}

int bsam_batch_run(bsam_batch* b) {
  if (!b) return BSAM_ERR_ARG;
  for (int guard = 0; guard < 1000000; ++guard) {
    int rc = bsam_batch_advance(b, 1 << 20);
    if (rc) return rc;
    rc = bsam_batch_sync(b);
    if (rc) return rc;
    if (running_slots(b) == 0 && !amr_waiting(b)) return BSAM_OK;
  }
  return fail(b, BSAM_ERR_STATE, "batch did not finish");
}

int bsam_batch_poll(bsam_batch* b, int* slots, int maxn) {
  if (!b) return BSAM_ERR_ARG;
  int n = 0;
  for (size_t s = 0; s < b->slots.size(); ++s) {
    if (!b->slots[s].used) continue;
    const int ph = ((volatile SlotOut*)b->h_out)[s].phase;
    if (ph == SLOT_DONE || ph == SLOT_FAILED) {
      if (slots && n < maxn) slots[n] = (int)s;
      ++n;
    }
  }
  return n;
}

int bsam_batch_slot_phase(bsam_batch* b, int slot, int* phase, int* steps_done) {
  if (!b || slot < 0 || slot >= (int)b->slots.size()) return BSAM_ERR_ARG;
  volatile SlotOut* o = b->h_out + slot;
  if (phase) *phase = b->slots[slot].used ? o->phase : SLOT_IDLE;
  if (steps_done) *steps_done = b->slots[slot].used ? o->step : 0;
  return BSAM_OK;
}

int bsam_batch_collect(bsam_batch* b, int slot, double* q, bsam_step_result* steps,
                       double* mass) {
  if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used)
    return BSAM_ERR_ARG;
  CU(cudaSetDevice(b->device));
  CU(cudaStreamSynchronize(b->stream));
  SlotPlan& S = b->slots[slot];
  const int ph = ((volatile SlotOut*)b->h_out)[slot].phase;
  if (ph != SLOT_DONE && ph != SLOT_FAILED) return fail(b, BSAM_ERR_STATE, "problem not finished");
  if (S.amr) {
    // A refined hierarchy: its state stays in its engine (read it there, or
    // through q / mass here); the slot is released.
    std::vector<StepLog> lg(S.nsteps);
    CU(cudaMemcpy(lg.data(), b->d_log + (int64_t)slot * BSAM_BATCH_MAX_STEPS,
                  sizeof(StepLog) * lg.size(), cudaMemcpyDeviceToHost));
    const int done = ((volatile SlotOut*)b->h_out)[slot].step;
    if (steps)
      for (int i = 0; i < S.nsteps; ++i) {
        steps[i].nvcycles = i < done ? lg[i].nv : 0;
        steps[i].converged = i < done ? lg[i].conv : 0;
        steps[i].residual = i < done ? lg[i].res : NAN;
      }
    int rc = BSAM_OK;
    if (q) {
      const EngineView& V = S.view;
      rc = bsam_gpu_get_field(S.eng, V.levels[0 - V.minlevel].patches[0], BSAM_FIELD_Q, q);
    }
    if (!rc && mass) rc = bsam_gpu_mass(S.eng, mass);
    if (S.ready) cudaEventDestroy(S.ready);
    S = SlotPlan{};  // its tiles are inactive records of the refined lists only
    ((volatile SlotOut*)b->h_out)[slot].phase = SLOT_IDLE;
    b->h_cfg[slot] = SlotCfg{};
    b->cfg_dirty = true;
    if (rc) return fail(b, rc, "reading the refined hierarchy's engine failed");
    return ph == SLOT_FAILED
               ? fail(b, BSAM_ERR_DIVERGED, "the problem failed: a residual was not finite or a "
                                            "regrid failed (bsam_batch_advance reported it)")
               : BSAM_OK;
  }
  const int nd = b->bp.ndims;
  const int rec_master = slot * RMAX + S.master;
  const DevPatch& M = S.recs[S.master];
  const SlotCfg& C = b->h_cfg[slot];
  if (q) {
    const int e0 = M.n[0] + 2, e1 = M.n[1] + 2, e2 = nd == 3 ? M.n[2] + 2 : 1;
    const size_t hcomp = (size_t)e0 * e1 * e2;
    for (int c = 0; c < 2; ++c)
      CU(cudaMemcpy2DAsync(q + c * hcomp, e0 * sizeof(double), M.q[c], M.sy * sizeof(double),
                           e0 * sizeof(double), (size_t)e1 * e2, cudaMemcpyDeviceToHost,
                           b->stream));
  }
  std::vector<StepLog> lg(S.prob.nsteps);
  CU(cudaMemcpyAsync(lg.data(), b->d_log + (int64_t)slot * BSAM_BATCH_MAX_STEPS,
                     sizeof(StepLog) * lg.size(), cudaMemcpyDeviceToHost, b->stream));
  if (mass) {
    const double hh = M.h;
    const double hd = nd == 2 ? hh * hh : hh * hh * hh;
    const int ni = C.ie - C.ib;
    const Item* items = b->lists[L_MASTER].d + C.ib;
    (void)rec_master;
    if (nd == 2)
      k_mass<double, 2><<<ni, dim3(32, TILE_Y), 0, b->stream>>>(b->d_pt, items, b->d_partials,
                                                                 b->d_status, ni, hd);
    else
      k_mass<double, 3><<<ni, dim3(32, TILE_Y), 0, b->stream>>>(b->d_pt, items, b->d_partials,
                                                                 b->d_status, ni, hd);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(b->h_status, b->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost,
                       b->stream));
  }
  CU(cudaStreamSynchronize(b->stream));
  const int done = ((volatile SlotOut*)b->h_out)[slot].step;
  if (steps)
    for (int i = 0; i < S.prob.nsteps; ++i) {
      if (i < done) {
        steps[i].nvcycles = lg[i].nv;
        steps[i].converged = lg[i].conv;
        steps[i].residual = lg[i].res;
      } else {
        steps[i].nvcycles = 0;
        steps[i].converged = 0;
        steps[i].residual = NAN;
      }
    }
  if (mass) *mass = b->h_status->mass;
  // Release: memory now, the slot once its tiles leave the lists.
  pool_free(b, S.off, S.bytes);
  S.used = false;
  S.stale = true;
  volatile SlotOut* o = b->h_out + slot;
  o->phase = SLOT_IDLE;
  int live = 0, dead = 0;
  for (auto& x : b->slots) {
    if (x.used) ++live;
    else if (x.stale) ++dead;
  }
  // Drop retired tiles once they outnumber the resident problems.
  if (dead > std::max(8, live)) compact(b);
  return ph == SLOT_FAILED ? fail(b, BSAM_ERR_DIVERGED, "residual is not finite") : BSAM_OK;
}

int bsam_batch_collect_many(bsam_batch* b, int n, const int* slots, double* const* qs,
                            bsam_step_result* const* steps, double* masses) {
  if (!b || n < 0 || (n > 0 && !slots)) return BSAM_ERR_ARG;
  if (n == 0) return BSAM_OK;
  CU(cudaSetDevice(b->device));
  for (int k = 0; k < n; ++k) {
    const int s = slots[k];
    if (s < 0 || s >= (int)b->slots.size() || !b->slots[s].used)
      return fail(b, BSAM_ERR_ARG, "slot not resident");
    if (b->slots[s].amr)
      return fail(b, BSAM_ERR_ARG, "refined hierarchies are collected one at a time");
    for (int k2 = 0; k2 < k; ++k2)
      if (slots[k2] == s) return fail(b, BSAM_ERR_ARG, "slot listed twice");
  }
  auto finished = [&]() {
    for (int k = 0; k < n; ++k) {
      const int ph = ((volatile SlotOut*)b->h_out)[slots[k]].phase;
      if (ph != SLOT_DONE && ph != SLOT_FAILED) return false;
    }
    return true;
  };
  // Without masses the read-back waits only for these slots to finish (their
  // phase in mapped host memory, written after everything else the control
  // kernel stores for them) and runs on the copy stream, beside any ticks
  // queued since.  The mass reduction shares the engine's partials with the
  // ticks, so with masses every queued tick is waited for first.
  const bool side = masses == nullptr;
  if (side) {
    while (!finished()) {
      const cudaError_t q = cudaStreamQuery(b->stream);
      if (q != cudaSuccess && q != cudaErrorNotReady)
        return fail(b, BSAM_ERR_CUDA, std::string("stream query: ") + cudaGetErrorString(q));
      if (q == cudaSuccess && !finished()) break;  // idle engine: the check below fails
      std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
  } else {
    CU(cudaStreamSynchronize(b->stream));
  }
  if (!finished()) return fail(b, BSAM_ERR_STATE, "problem not finished");
  cudaStream_t cs = side ? b->xstream : b->stream;
  const int nd = b->bp.ndims;
  // Step logs: one launch writes every slot's log into page-locked staging;
  // masses: the per-slot reduction, each total copied into staging.
  // Root states wanted: packed into the transfer buffer by one launch, then
  // one contiguous copy per problem into the caller's buffer.
  std::vector<size_t> xo((size_t)n + 1, 0);
  int nq = 0;
  for (int k = 0; k < n; ++k) {
    const SlotPlan& S = b->slots[slots[k]];
    const DevPatch& M = S.recs[S.master];
    const size_t w = (qs && qs[k])
                         ? 2 * (size_t)(M.n[0] + 2) * (M.n[1] + 2) * (nd == 3 ? M.n[2] + 2 : 1)
                         : 0;
    nq += w ? 1 : 0;
    xo[k + 1] = xo[k] + w;
  }
  double* xfer = nullptr;
  if (nq && !(xfer = xfer_reserve(b, &b->d_xout, &b->xout_words, xo[n])))
    return fail(b, BSAM_ERR_NOMEM, "transfer buffer allocation failed");
  char* st = stage_alloc(b, sizeof(RowsTask) * n + sizeof(WordSpan) * n +
                                sizeof(StepLog) * BSAM_BATCH_MAX_STEPS * n +
                                sizeof(DevStatus) * n + 64);
  if (!st) return fail(b, BSAM_ERR_NOMEM, "pinned staging allocation failed");
  RowsTask* rows = reinterpret_cast<RowsTask*>(st);
  WordSpan* spans = reinterpret_cast<WordSpan*>(rows + n);
  StepLog* logs = reinterpret_cast<StepLog*>(spans + n);
  DevStatus* stat = reinterpret_cast<DevStatus*>(logs + (size_t)BSAM_BATCH_MAX_STEPS * n);
  int64_t maxw = 1;
  for (int k = 0; k < n; ++k) {
    const SlotPlan& S = b->slots[slots[k]];
    const int64_t nw = (int64_t)(sizeof(StepLog) * S.prob.nsteps / 8);
    spans[k] = WordSpan{reinterpret_cast<const uint64_t*>(b->d_log +
                                                          (int64_t)slots[k] * BSAM_BATCH_MAX_STEPS),
                        reinterpret_cast<uint64_t*>(logs + (size_t)k * BSAM_BATCH_MAX_STEPS), nw};
    maxw = std::max(maxw, nw);
  }
  k_word_spans<<<dim3((unsigned)((maxw + 255) / 256), n), 256, 0, cs>>>(spans);
  if (nq) {
    int nt = 0;
    int64_t maxr = 0;
    std::vector<int> which;
    which.reserve(nq);
    for (int k = 0; k < n; ++k) {
      if (xo[k + 1] == xo[k]) continue;
      const SlotPlan& S = b->slots[slots[k]];
      const DevPatch& M = S.recs[S.master];
      const int64_t nrow = (int64_t)(M.n[1] + 2) * (nd == 3 ? M.n[2] + 2 : 1);
      rows[nt++] = RowsTask{xfer + xo[k], {static_cast<double*>(M.q[0]), static_cast<double*>(M.q[1])},
                            nrow, M.sy, M.n[0] + 2, 0};
      maxr = std::max(maxr, 2 * nrow);
      which.push_back(k);
    }
    const unsigned gr = (unsigned)std::max<int64_t>(1, std::min<int64_t>((maxr + 7) / 8, 64));
    k_rows_list<false><<<dim3(gr, nt), 256, 0, cs>>>(rows);
    for (int k : which)
      CU(cudaMemcpyAsync(qs[k], xfer + xo[k], sizeof(double) * (xo[k + 1] - xo[k]),
                         cudaMemcpyDeviceToHost, cs));
  }
  for (int k = 0; k < n; ++k) {
    const SlotPlan& S = b->slots[slots[k]];
    const DevPatch& M = S.recs[S.master];
    if (masses) {
      const SlotCfg& C = b->h_cfg[slots[k]];
      const double hh = M.h;
      const double hd = nd == 2 ? hh * hh : hh * hh * hh;
      const int ni = C.ie - C.ib;
      const Item* items = b->lists[L_MASTER].d + C.ib;
      if (nd == 2)
        k_mass<double, 2><<<ni, dim3(32, TILE_Y), 0, b->stream>>>(b->d_pt, items, b->d_partials,
                                                                   b->d_status, ni, hd);
      else
        k_mass<double, 3><<<ni, dim3(32, TILE_Y), 0, b->stream>>>(b->d_pt, items, b->d_partials,
                                                                   b->d_status, ni, hd);
      CU(cudaMemcpyAsync(stat + k, b->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost,
                         b->stream));
    }
  }
  CU(cudaGetLastError());
  stage_commit(b, cs);
  CU(cudaStreamSynchronize(cs));
  int rc = BSAM_OK;
  for (int k = 0; k < n; ++k) {
    const int s = slots[k];
    SlotPlan& S = b->slots[s];
    const int done = ((volatile SlotOut*)b->h_out)[s].step;
    const StepLog* lg = logs + (size_t)k * BSAM_BATCH_MAX_STEPS;
    if (steps && steps[k])
      for (int i = 0; i < S.prob.nsteps; ++i) {
        steps[k][i].nvcycles = i < done ? lg[i].nv : 0;
        steps[k][i].converged = i < done ? lg[i].conv : 0;
        steps[k][i].residual = i < done ? lg[i].res : NAN;
      }
    if (masses) masses[k] = stat[k].mass;
    if (((volatile SlotOut*)b->h_out)[s].phase == SLOT_FAILED) rc = BSAM_ERR_DIVERGED;
    pool_free(b, S.off, S.bytes);
    S.used = false;
    S.stale = true;
    ((volatile SlotOut*)b->h_out)[s].phase = SLOT_IDLE;
  }
  int live = 0, dead = 0;
  for (auto& x : b->slots) {
    if (x.used) ++live;
    else if (x.stale) ++dead;
  }
  if (dead > std::max(8, live)) compact(b);
  return rc == BSAM_OK ? BSAM_OK : fail(b, rc, "a residual is not finite");
}

int bsam_batch_get_stream(bsam_batch* b, void** stream) {
  if (!b || !stream) return BSAM_ERR_ARG;
  *stream = (void*)b->stream;
  return BSAM_OK;
}

int bsam_batch_get_stats(bsam_batch* b, bsam_batch_stats* s) {
  if (!b || !s) return BSAM_ERR_ARG;
  cudaSetDevice(b->device);
  BatchCtl c{};
  if (cudaMemcpy(&c, b->d_ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(b, BSAM_ERR_CUDA, "stats read failed");
  bsam_batch_stats o = b->st;
  o.ticks = c.ticks;
  o.kernels_per_tick = b->kernels_per_tick;
  o.launches = c.ticks * b->kernels_per_tick;
  o.pool_used = (int64_t)b->pool_used;
  o.pool_bytes = (int64_t)b->pool_bytes;
  o.resident = 0;
  for (auto& x : b->slots) o.resident += x.used ? 1 : 0;
  o.running = running_slots(b);
  *s = o;
  return BSAM_OK;
}

}  // extern "C"
