// bsam_noalloc.cu -- residual norm of one patch without any device allocation.
//
// Some callers cannot allocate device memory when they need this number: a
// host whose device memory is already handed to its own pool (for example a
// Fortran code with one preallocated arena, or PyTorch's caching allocator
// holding the free memory), or a time-step loop that must not pay the
// implicit device-wide synchronisation of cudaMalloc/cudaFree.  For them,
// bsam_gpu_resid_norm_noalloc computes the ErrorAFAS residual norm
// (errortype 1, lib/afasroutines.f90:108-221) of fields that live in the
// caller's own device memory, using a fixed scratch array compiled into the
// library instead of allocated storage.
//
// Scratch: g_noalloc_scratch below, a file-scope __device__ array.  Every GPU
// that loads this library holds it (NOALLOC_SCRATCH_BYTES) until the process
// exits.  All calls share it, so calls whose kernels overlap on the GPU (two
// host threads, or two streams without ordering between them) race on it and
// give wrong results; order such calls on one stream.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/bsam_gpu.h"
#include "bsam_types.h"
#include "kernels.cuh"

using namespace bsam;

namespace {

// One partial sum per CTA (tile of 64 x 4 x 1 cells) plus the ticket of the
// last-block-done reduction in the trailing 256 bytes.
constexpr int NOALLOC_MAX_TILES = BSAM_NOALLOC_MAX_TILES;
constexpr int NOALLOC_TAIL_DOUBLES = 32;
constexpr size_t NOALLOC_SCRATCH_BYTES =
    sizeof(double) * (NOALLOC_MAX_TILES + NOALLOC_TAIL_DOUBLES);

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_MAX_TILES +
                                                          NOALLOC_TAIL_DOUBLES];
static_assert(sizeof(g_noalloc_scratch) == NOALLOC_SCRATCH_BYTES &&
                  NOALLOC_SCRATCH_BYTES <= 512 * 1024 + 256,
              "the scratch array is meant to stay near 512 KiB");

// Device address of g_noalloc_scratch per device.  In host code the symbol
// name is only a host-side stand-in, never a device address, so the address
// is looked up once per device with cudaGetSymbolAddress.
constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_scratch_addr[kMaxDevices] = {nullptr};

int scratch_for_device(int device, double** out) {
  if (device < 0 || device >= kMaxDevices) return BSAM_ERR_NODEVICE;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p)
      return BSAM_ERR_CUDA;
    g_scratch_addr[device] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[device];
  return BSAM_OK;
}

// Variant of k_resid_norm that reads the caller's Fortran-layout arrays and
// reduces through the static scratch.  The tile of a CTA is derived from
// blockIdx in the same x-fastest order as the library's work lists, so the
// partial sums are combined in the same order as bsam_gpu_multigrid_iterations.
template <int D>
__global__ void __launch_bounds__(BLOCK_THREADS)
    k_resid_norm_noalloc(DevPatch P, const double* __restrict__ fbase, int64_t fsy,
                         int64_t fsz, int64_t fcomp, int tiles_x, int tiles_y,
                         double* __restrict__ scratch, double denom, double* __restrict__ out) {
  const int b = blockIdx.x;
  const int tx = b % tiles_x, ty = (b / tiles_x) % tiles_y, tz = b / (tiles_x * tiles_y);
  const int j = ty * TILE_Y + threadIdx.y + 1;
  const int k = (D == 3) ? tz + 1 : 0;
  const int i0 = (tx * 32 + threadIdx.x) * 2 + 1;
  const double* q0 = static_cast<const double*>(P.q[0]);
  const double* q1 = static_cast<const double*>(P.q[1]);
  double acc = 0.0;
  if (j <= P.n[1]) {
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      const int i = i0 + t;
      if (i <= P.n[0]) {
        Problem::Stencil<double, D> s;
        load_stencil<double, D>(P, q0, q1, cidx(P, i, j, k), s);
        double o0, o1;
        Problem::OperatorCell<double, D>(s, P.tmp1, P.tmp2, P.alpha, o0, o1);
        const int64_t fc = (int64_t)(i - 1) + (int64_t)(j - 1) * fsy +
                           (int64_t)(D == 3 ? k - 1 : 0) * fsz;
        const double r0 = fbase[fc] - o0;
        const double r1 = fbase[fc + fcomp] - o1;
        acc += r0 * r0 + r1 * r1;
      }
    }
  }
  const double bs = block_sum(acc);
  double total;
  uint32_t* ticket = reinterpret_cast<uint32_t*>(scratch + NOALLOC_MAX_TILES);
  if (last_block_total(bs, scratch, ticket, (int)gridDim.x, total)) {
    out[0] = sqrt(total / denom);
    out[1] = total;
  }
}

}  // namespace

extern "C" int bsam_gpu_resid_norm_noalloc(int device, int ndims, const int32_t* mx, double dx,
                                           double dt, double eps, double alpha, const double* q,
                                           const double* f, double* out, void* stream) {
  if ((ndims != 2 && ndims != 3) || !mx || !q || !f || !out || !(dx > 0.0))
    return BSAM_ERR_ARG;
  int64_t n[3] = {1, 1, 1};
  for (int d = 0; d < ndims; ++d) {
    if (mx[d] <= 0) return BSAM_ERR_ARG;
    n[d] = mx[d];
  }
  const int64_t tiles_x = (n[0] + TILE_X - 1) / TILE_X;
  const int64_t tiles_y = (n[1] + TILE_Y - 1) / TILE_Y;
  const int64_t tiles = tiles_x * tiles_y * n[2];
  if (tiles > NOALLOC_MAX_TILES) return BSAM_ERR_TOO_LARGE;

  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return BSAM_ERR_NODEVICE;
  if (cudaSetDevice(device) != cudaSuccess) return BSAM_ERR_NODEVICE;
  double* scratch = nullptr;
  int rc = scratch_for_device(device, &scratch);
  if (rc == BSAM_OK) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DevPatch P{};
    P.ndims = ndims;
    for (int d = 0; d < 3; ++d) P.n[d] = (int32_t)n[d];
    P.sy = n[0] + 2;
    P.sz = ndims == 3 ? (n[0] + 2) * (n[1] + 2) : 0;
    const int64_t qcomp = (n[0] + 2) * (n[1] + 2) * (ndims == 3 ? n[2] + 2 : 1);
    P.q[0] = const_cast<double*>(q);
    P.q[1] = const_cast<double*>(q) + qcomp;
    // Operator constants computed as in problem.f90:246-248.
    const double h2 = dx * dx;
    P.h = dx;
    P.alpha = alpha;
    P.tmp1 = dt / h2;
    P.tmp2 = eps * eps / h2;
    const double denom = (double)(2 * n[0] * n[1] * n[2]);
    // The ticket must start at zero; the partials are written before read.
    uint32_t* ticket = reinterpret_cast<uint32_t*>(scratch + NOALLOC_MAX_TILES);
    if (cudaMemsetAsync(ticket, 0, sizeof(uint32_t), s) != cudaSuccess) {
      rc = BSAM_ERR_CUDA;
    } else {
      const dim3 block(32, TILE_Y, 1);
      const int64_t fsy = n[0], fsz = n[0] * n[1], fcomp = n[0] * n[1] * n[2];
      if (ndims == 2)
        k_resid_norm_noalloc<2><<<(unsigned)tiles, block, 0, s>>>(
            P, f, fsy, fsz, fcomp, (int)tiles_x, (int)tiles_y, scratch, denom, out);
      else
        k_resid_norm_noalloc<3><<<(unsigned)tiles, block, 0, s>>>(
            P, f, fsy, fsz, fcomp, (int)tiles_x, (int)tiles_y, scratch, denom, out);
      if (cudaGetLastError() != cudaSuccess) rc = BSAM_ERR_CUDA;
    }
  }
  cudaSetDevice(prev);
  return rc;
}
