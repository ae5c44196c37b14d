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

// Grid-wide sums of NV values that stay deterministic on any number of
// CTAs: every CTA reduces its values with block_sum and stores the results
// as part[v * gridDim.x + blockIdx.x]; the CTA that finishes last (counted
// on *counter) sums the partials of each value in index order with a fixed
// thread assignment, so the totals do not depend on which CTA that is.
// Returns true in the last CTA, whose thread 0 then holds the totals in
// tot; the last CTA also resets *counter for the next launch.  All threads
// of every CTA must call it.  `sh` holds blockDim/32 + 1 doubles.
template <int NV>
__device__ __forceinline__ bool grid_sums_last(const double (&v)[NV], double *part, unsigned *counter, double *sh,
                                               double (&tot)[NV]) {
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthreads = blockDim.x * blockDim.y * blockDim.z;
  const unsigned G = gridDim.x * gridDim.y * gridDim.z;
  const unsigned b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
#pragma unroll
  for (int i = 0; i < NV; i++) {
    const double s = block_sum(v[i], sh);
    if (tid == 0) part[(size_t)i * G + b] = s;
  }
  __shared__ int last;
  if (tid == 0) {
    __threadfence();  // this CTA's partials are visible before it is counted
    last = (atomicAdd(counter, 1u) == G - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
#pragma unroll
  for (int i = 0; i < NV; i++) {
    double acc = 0.0;
    for (unsigned c = tid; c < G; c += nthreads) acc += __ldcg(part + (size_t)i * G + c);
    tot[i] = block_sum(acc, sh);
  }
  if (tid == 0) *counter = 0u;
  return true;
}

// Reduce `nvals` independent partial arrays part[v*stride + b], b < nb, into
// out[v] = (mult * sum_b part[...]) / div (one CTA of 1024 threads).
__global__ void k_finalize_sums(const double *__restrict__ part, size_t stride, int nb, int nvals, double mult,
                                double div, double *out);

}  // namespace he4
