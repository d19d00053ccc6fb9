// blas.cu -- precision conversion and deterministic FP64 reductions.
//
// Reductions write one partial sum per block; finish_sum adds the partials
// in a fixed order, so every result is bit-reproducible run to run.
#include "thr_common.cuh"
#include "thr_kernels.h"

namespace thr {

namespace {
constexpr int kRedThreads = 256;

inline int red_blocks(size_t n) {
  size_t b = (n + kRedThreads * 4 - 1) / (kRedThreads * 4);
  if (b > device_sms() * 8) b = device_sms() * 8;
  if (b < 1) b = 1;
  return (int)b;
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double sh[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? sh[threadIdx.x] : 0.0;
  if (w == 0) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

template <class S>
__global__ void k_norm2(const S* a, size_t n, double* partials) {
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    auto v = Sto<S>::ld(a, i);
    double x = (double)v.x, y = (double)v.y;
    acc += x * x + y * y;
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

template <class S>
__global__ void k_redot(const S* a, const S* b, size_t n, double* partials) {
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    auto u = Sto<S>::ld(a, i);
    auto v = Sto<S>::ld(b, i);
    acc += (double)u.x * (double)v.x + (double)u.y * (double)v.y;
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

__global__ void k_finish(const double* partials, int np, double* out) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) acc += partials[i];
  acc = block_sum(acc);
  if (threadIdx.x == 0) *out = acc;
}

template <class Sd, class Ss>
__global__ void k_convert(Sd* d, const Ss* s, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    auto v = Sto<Ss>::ld(s, i);
    Sto<Sd>::st(d, i, typename Sto<Sd>::C{(typename Sto<Sd>::R)v.x, (typename Sto<Sd>::R)v.y});
  }
}

__global__ void k_axpy(double2* y, const double2* x, double a, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = y[i] + a * x[i];
}
__global__ void k_scale_copy(double2* y, const double2* x, double a, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = a * x[i];
}

inline unsigned ew_grid(size_t n) {
  size_t b = (n + 255) / 256;
  if (b > device_sms() * 16) b = device_sms() * 16;
  return (unsigned)(b ? b : 1);
}
}  // namespace

template <class S>
int norm2_partials(const S* a, size_t n, double* partials, cudaStream_t st) {
  int nb = red_blocks(n);
  k_norm2<S><<<nb, kRedThreads, 0, st>>>(a, n, partials);
  return nb;
}
template <class S>
int redot_partials(const S* a, const S* b, size_t n, double* partials, cudaStream_t st) {
  int nb = red_blocks(n);
  k_redot<S><<<nb, kRedThreads, 0, st>>>(a, b, n, partials);
  return nb;
}
void finish_sum(const double* partials, int np, double* out, cudaStream_t st) {
  k_finish<<<1, 1024, 0, st>>>(partials, np, out);
}

template <class Sd, class Ss>
void convert(Sd* dst, const Ss* src, size_t n, cudaStream_t st) {
  k_convert<Sd, Ss><<<ew_grid(n), 256, 0, st>>>(dst, src, n);
}
void axpy_d(double2* y, const double2* x, double a, size_t n, cudaStream_t st) {
  k_axpy<<<ew_grid(n), 256, 0, st>>>(y, x, a, n);
}
void scale_copy_d(double2* y, const double2* x, double a, size_t n, cudaStream_t st) {
  k_scale_copy<<<ew_grid(n), 256, 0, st>>>(y, x, a, n);
}

template int norm2_partials<double2>(const double2*, size_t, double*, cudaStream_t);
template int norm2_partials<float2>(const float2*, size_t, double*, cudaStream_t);
template int norm2_partials<__nv_bfloat162>(const __nv_bfloat162*, size_t, double*, cudaStream_t);
template int redot_partials<double2>(const double2*, const double2*, size_t, double*, cudaStream_t);
template int redot_partials<float2>(const float2*, const float2*, size_t, double*, cudaStream_t);
template void convert<float2, double2>(float2*, const double2*, size_t, cudaStream_t);
template void convert<double2, float2>(double2*, const float2*, size_t, cudaStream_t);
template void convert<__nv_bfloat162, double2>(__nv_bfloat162*, const double2*, size_t, cudaStream_t);
template void convert<double2, __nv_bfloat162>(double2*, const __nv_bfloat162*, size_t, cudaStream_t);
template void convert<__nv_bfloat162, float2>(__nv_bfloat162*, const float2*, size_t, cudaStream_t);
template void convert<float2, __nv_bfloat162>(float2*, const __nv_bfloat162*, size_t, cudaStream_t);

}  // namespace thr
