// stats.cuh -- after-step statistics over a whole hierarchy.
//
// AfterStepStatistics (lib/bsamroutines.f90:893-937) calls AfterStep2D/3D
// (problem.f90:102-134, 398-424) on every patch, finest level first:
//   level 0:  integral(1) += h^d sum(c);  integral(2) += Energy2D(c, h)  (2D)
//   level >0: integral(1) += h^d sum(c) - (2h)^d sum(parent c over the footprint)
//             integral(2) += Energy2D(c, h) - Energy2D(parent c over the
//                            footprint and its ring, 2h)                   (2D)
// Each sum is a "term": a box of one patch's interior and what is summed over
// it -- c, Ff(c), or Energy2D's squared differences (which read one cell
// beyond the box).  A term's rows are split over CTAs; each CTA writes one
// partial, and the host adds the partials of a term in row order.
#pragma once
#include "kernels.cuh"

namespace bsam {

enum StatKind : int32_t { STAT_SUM = 0, STAT_FF = 1, STAT_GRAD2 = 2 };

struct StatBlock {
  int32_t patch, kind;
  int32_t lo[3], hi[3];  // the term's box, patch index space
  int32_t row0, row1;    // rows (j, k) of the box this CTA sums, [row0, row1)
};

template <int D>
__global__ void __launch_bounds__(256)
    k_stats(const DevPatch* __restrict__ PT, const StatBlock* __restrict__ blocks,
            double* __restrict__ partials) {
  const StatBlock b = blocks[blockIdx.x];
  const DevPatch P = PT[b.patch];
  const double* c = fld<double>(P.q[0]);
  const int ny = b.hi[1] - b.lo[1] + 1;
  const double alpha = P.alpha;
  double acc = 0.0;
  for (int r = b.row0; r < b.row1; ++r) {
    const int j = b.lo[1] + r % ny;
    const int k = D == 3 ? b.lo[2] + r / ny : 0;
    for (int i = b.lo[0] + (int)threadIdx.x; i <= b.hi[0]; i += blockDim.x) {
      const double x = c[cidx(P, i, j, k)];
      if (b.kind == STAT_SUM) {
        acc += x;
      } else if (b.kind == STAT_FF) {
        acc += Problem::Ff(x, alpha);
      } else {
        const double a = c[cidx(P, i + 1, j, k)] - x, e = x - c[cidx(P, i - 1, j, k)];
        const double u = c[cidx(P, i, j + 1, k)] - x, w = x - c[cidx(P, i, j - 1, k)];
        acc += a * a + e * e + u * u + w * w;
      }
    }
  }
  const double s = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

}  // namespace bsam
