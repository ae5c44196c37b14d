// reduce.cuh -- deterministic FP64 block reductions.
//
// Every reduction is a fixed tree: warp shuffles, then one warp over the
// per-warp sums, then a single CTA over the per-block partials in index
// order.  Results therefore do not depend on scheduling.
#pragma once
#include "common.cuh"

namespace he4 {

// Sum of v over the block; the result is valid in thread 0.
// `sh` must hold blockDim/32 doubles.
__device__ __forceinline__ double block_sum(double v, double *sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nthreads = blockDim.x * blockDim.y * blockDim.z;
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int lane2 = tid & 31, warp2 = tid >> 5;
  (void)lane;
  (void)warp;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (lane2 == 0) sh[warp2] = v;
  __syncthreads();
  const int nw = (nthreads + 31) >> 5;
  double r = 0.0;
  if (warp2 == 0) {
    r = (lane2 < nw) ? sh[lane2] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  return r;
}

// Reduce `nvals` independent partial arrays part[v*stride + b], b < nb, into
// out[v] = (mult * sum_b part[...]) / div (one CTA of 1024 threads).
__global__ void k_finalize_sums(const double *__restrict__ part, size_t stride, int nb, int nvals, double mult,
                                double div, double *out);

}  // namespace he4
