// thr_reduce.cuh -- deterministic block reductions shared by the solver kernels.
#pragma once
#include <cuda_runtime.h>

namespace thr {

// Sum of partials[0..n) by one block; every thread receives the total.  The
// order of additions is fixed by (n, blockDim), so results are reproducible.  Each
// thread issues up to eight of its loads before it adds them (in index order), so
// that their latencies overlap instead of adding up.
__device__ __forceinline__ double block_sum_partials(const double* partials, int n) {
  __shared__ double sh[33];
  double v = 0.0;
  constexpr int kU = 8;
  const int stride = blockDim.x;
  int i = threadIdx.x;
  for (; i + (kU - 1) * stride < n; i += kU * stride) {
    double x[kU];
#pragma unroll
    for (int u = 0; u < kU; u++) x[u] = partials[i + u * stride];
#pragma unroll
    for (int u = 0; u < kU; u++) v += x[u];
  }
  for (; i < n; i += stride) v += partials[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    const int nw = (blockDim.x + 31) >> 5;
    v = threadIdx.x < nw ? sh[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) sh[32] = v;
  }
  __syncthreads();
  v = sh[32];
  __syncthreads();
  return v;
}

// block-wide sum of one value per thread; thread 0 writes partials[blockIdx.x]
__device__ __forceinline__ void block_write_partial(double v, double* partials) {
  __shared__ double sh[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    const int nw = (blockDim.x + 31) >> 5;
    v = threadIdx.x < nw ? sh[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) partials[blockIdx.x] = v;
  }
}

}  // namespace thr
