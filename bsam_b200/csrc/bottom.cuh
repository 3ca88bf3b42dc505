// bottom.cuh -- the coarse end of the V-cycle in one launch.
//
// Below a few thousand cells a level is far too small to fill the GPU, and a
// launch per colour pass and per transfer makes the coarse levels of a
// V-cycle launch-latency bound.  k_bottom runs AFASVcycle (afas:488-521) for
// a whole chain of small uniform levels -- from the chain's top patch down to
// the coarsest level and back -- inside one CTA, with __syncthreads between
// the phases the reference separates (every colour pass, restriction, coarse
// load, correction).  The per-cell arithmetic is the same device code as the
// grid kernels, so the results are identical.  One CTA per chain: a batch of
// independent problems runs its bottoms side by side in one launch.
#pragma once
#include "kernels.cuh"

namespace bsam {

constexpr int BOTTOM_THREADS = 512;
constexpr int BOTTOM_MAX_CELLS = 4096;  // largest level handled by k_bottom
constexpr int BOTTOM_MAX_DEPTH = 16;

template <class T, int D>
__device__ __forceinline__ void block_relax(const DevPatch& P, int nu) {
  const int npx = (P.n[0] + 1) / 2;
  const int total = npx * P.n[1] * (D == 3 ? P.n[2] : 1);
  for (int pass = 0; pass < 2 * nu; ++pass) {
    const int color = pass & 1;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
      const int px = idx % npx, rest = idx / npx;
      const int j = rest % P.n[1] + 1;
      const int k = (D == 3) ? rest / P.n[1] + 1 : 0;
      const int i0 = 2 * px + 1;
      const int i = i0 + ((i0 + j + k + color) & 1);
      if (i <= P.n[0]) relax_cell<T, D>(P, i, j, k);
    }
    __syncthreads();
  }
}

template <class T, int D>
__device__ __forceinline__ void block_restrict_load(const DevPatch& C, const DevPatch& P) {
  const int total = C.cn[0] * C.cn[1] * (D == 3 ? C.cn[2] : 1);
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int ic = idx % C.cn[0] + 1, rest = idx / C.cn[0];
    const int jc = rest % C.cn[1] + 1;
    const int kc = (D == 3) ? rest / C.cn[1] + 1 : 0;
    restrict_cell<T, T, D>(C, P, ic, jc, kc);
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int ic = idx % C.cn[0] + 1, rest = idx / C.cn[0];
    const int jc = rest % C.cn[1] + 1;
    const int kc = (D == 3) ? rest / C.cn[1] + 1 : 0;
    coarse_load_cell<T, T, D>(C, P, ic, jc, kc);
  }
  __syncthreads();
}

template <class T, int D>
__device__ __forceinline__ void block_correct(const DevPatch& C, const DevPatch& P) {
  const int total = C.n[0] * C.n[1] * (D == 3 ? C.n[2] : 1);
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int I = idx % C.n[0] + 1, rest = idx / C.n[0];
    const int J = rest % C.n[1] + 1;
    const int K = (D == 3) ? rest / C.n[1] + 1 : 0;
    correct_cell<T, T, D>(C, P, I, J, K);
  }
  __syncthreads();
}

// AFASVcycle from `top` down its parent links to the coarsest level and back,
// by the whole CTA.  chain / depth: the caller's shared scratch.
template <class T, int D>
__device__ __forceinline__ void bottom_chain(const DevPatch* __restrict__ PT, int top, int nu,
                                             int* chain, int& depth) {
  __syncthreads();  // chain[] of a previous call is no longer read
  if (threadIdx.x == 0) {
    int d = 0;
    for (int p = top; p >= 0 && d < BOTTOM_MAX_DEPTH; p = PT[p].parent) chain[d++] = p;
    depth = d;
  }
  __syncthreads();
  const int nd = depth;
  // Down: pre-smoothing, restriction and coarse load (afas:499-509).
  for (int l = 0; l < nd; ++l) {
    const DevPatch P = PT[chain[l]];
    block_relax<T, D>(P, nu);
    if (l + 1 < nd) {
      const DevPatch Q = PT[chain[l + 1]];
      block_restrict_load<T, D>(P, Q);
    }
  }
  // Up: correction and post-smoothing (afas:513-517).
  for (int l = nd - 2; l >= 0; --l) {
    const DevPatch P = PT[chain[l]];
    const DevPatch Q = PT[chain[l + 1]];
    block_correct<T, D>(P, Q);
    block_relax<T, D>(P, nu);
  }
}

// tops[b]: the top patch of chain b; the chain follows parent links down to
// the coarsest level.  nu = nsmoothingpasses.  Chains whose top is inactive
// (finished batch slots) are skipped.
template <class T, int D>
__global__ void __launch_bounds__(BOTTOM_THREADS)
    k_bottom(const DevPatch* __restrict__ PT, const int* __restrict__ tops, int nu) {
  __shared__ int chain[BOTTOM_MAX_DEPTH];
  __shared__ int depth;
  const int top = tops[blockIdx.x];
  if (!PT[top].active) return;
  bottom_chain<T, D>(PT, top, nu, chain, depth);
}

}  // namespace bsam
