// engine_view.h -- what the batched engine reads of a single-problem engine
// whose time steps it runs (bsam_batch_submit_amr).  Internal to the
// library: both engines are compiled into the same shared object.
//
// A refined hierarchy keeps its fields in its own engine (bsam_gpu.cu) and
// is regridded there by the native AMR driver (bsam_host.cpp) before every
// time step.  The batch copies the engine's patch records into its own
// table (same field pointers) and runs the step's MultigridIterations in
// the launches it issues for all its problems.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "amr.cuh"
#include "bsam_types.h"

struct bsam_gpu;
struct bsam_amr;

namespace bsam {

struct EngineLevelView {
  int level = 0;
  bool amr = false;   // above the root: SetGhost by interpolation + overlap + SetBC
  bool snap = false;  // a parent level its children do not cover (full q -> qs copy)
  std::vector<int> patches;       // records of the level, ApplyOnLevel order
  std::vector<OverlapCopy> ovl;   // refined levels: GhostOverlap transfers by destination
  std::vector<int2> range;        // per entry of patches: {first, count} into ovl
};

struct EngineView {
  int ndims = 2, minlevel = 0, finestlevel = 0;
  int nsmoothingpasses = 2, maxvcycles = 1;
  bool mixed = false;
  double qerrortol = 0.0;
  double denom = 1.0;                 // nrvars * cells of the finest level
  std::vector<DevPatch> recs;         // the engine's records (indices are record numbers)
  std::vector<EngineLevelView> levels;  // index level - minlevel
  std::vector<int> masters;           // finest-level records, in ErrorAFAS's order
};

// Fills v from the hierarchy set on h (BSAM_ERR_STATE without one).
int engine_view(bsam_gpu* h, EngineView& v);

// The start of MultigridIterations (afas:47-64), queued on the engine's
// stream: FillDown(solution) over the refined levels, then
// GetSourceFunction + UpdateSourceFunction on the levels >= root.  FP64 form.
int engine_prologue(bsam_gpu* h);

cudaStream_t engine_stream(bsam_gpu* h);
int engine_device(bsam_gpu* h);

// The engine a native AMR driver steps (bsam_amr_create's h).
bsam_gpu* amr_engine(bsam_amr* a);

}  // namespace bsam
