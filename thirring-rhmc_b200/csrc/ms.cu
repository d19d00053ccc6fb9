// ms.cu -- multishift CG (multishift_module.F90:13-284 and :289-534).
//
// Device-resident recurrences: the per-shift zeta/omega/gamma scalars, the
// convergence flags and the active window [minishift, maxishift] are kept in
// device memory and advanced by one-thread kernels; vector kernels read their
// coefficients from there.  The shift update touches every active shift in
// one pass over r and p (r and p are read once per iteration, not once per
// shift).  V = double2 gives the FP64 solver, V = float2 the reference's
// single-precision solver (FP32 vectors and FP32-rounded coefficients, FP64
// scalars and FP64 accumulation of FP32 terms as reduce_real_dp5d does).
#include <cmath>

#include "ctx.h"
#include "ms.h"
#include "solver.h"
#include "thr_reduce.cuh"

namespace thr {

namespace {
constexpr int kThreads = 256;

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

template <class V> struct VT;
template <> struct VT<double2> {
  using R = double;
  // |z|^2 term and Re(conj(a) b) term in the working precision
  static __device__ __forceinline__ double abs2(double2 a) { return a.x * a.x + a.y * a.y; }
  static __device__ __forceinline__ double redot(double2 a, double2 b) { return a.x * b.x + a.y * b.y; }
  static __device__ __forceinline__ double cast(double v) { return v; }
};
template <> struct VT<float2> {
  using R = float;
  // FP32 terms summed into FP64 (reductions.F90:6-32)
  static __device__ __forceinline__ double abs2(float2 a) { return (double)(a.x * a.x + a.y * a.y); }
  static __device__ __forceinline__ double redot(float2 a, float2 b) { return (double)(a.x * b.x + a.y * b.y); }
  static __device__ __forceinline__ float cast(double v) { return (float)v; }  // real(omega) etc.
};

template <class V>
__global__ void k_norm2(const MsState* ms, const V* a, size_t n, double* partials) {
  if (ms && ms->done) return;
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    acc += VT<V>::abs2(a[i]);
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}
template <class V>
__global__ void k_redot(const MsState* ms, const V* a, const V* b, size_t n, double* partials) {
  if (ms->done) return;
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    acc += VT<V>::redot(a[i], b[i]);
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

__global__ void k_ms_init(MsState* ms, const double* partials, int np) {
  const double d = block_sum_partials(partials, np);  // :73
  if (threadIdx.x == 0) ms->delta = d;
}

// iteration start + alpha: :104, :118-135 (one block; shifts in parallel)
__global__ void k_ms_alpha(MsState* ms, const double* partials, int np) {
  if (ms->done) return;
  const double alpha = block_sum_partials(partials, np);
  if (threadIdx.x == 0) ms_alpha_scalar(ms, alpha);
  __syncthreads();
  const int k = ms->lo + threadIdx.x;
  if (k <= ms->hi) ms_alpha_shift(ms, k);
}

// r = r + omega*s (:137) fused with lambda = |r|^2 (:138)
template <class V>
__global__ void k_ms_rupdate(const MsState* ms, V* r, const V* s, size_t n, double* partials) {
  if (ms->done) return;
  using R = typename VT<V>::R;
  const R om = VT<V>::cast(ms->omega);
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    V v = r[i] + om * s[i];
    r[i] = v;
    acc += VT<V>::abs2(v);
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

// :143, :148-150
__global__ void k_ms_lambda(MsState* ms, const double* partials, int np) {
  if (ms->done) return;
  const double lambda = block_sum_partials(partials, np);
  if (threadIdx.x == 0) ms_lambda_scalar(ms, lambda);
  __syncthreads();
  const int k = ms->lo + threadIdx.x;
  if (k <= ms->hi) ms_lambda_shift(ms, k);
}

// p = r + gammag*p (:145) and, for every shift in the window,
// out -= omegas*sf ; sf = sf*gammas + r*zeta_iii (:155-176)
template <class V>
__global__ void k_ms_pshift(const MsState* ms, V* p, const V* r, V* out, V* sf, size_t n, size_t stride) {
  if (ms->done) return;
  using R = typename VT<V>::R;
  const R gg = VT<V>::cast(ms->gammag);
  const int lo = ms->lo, hi = ms->hi;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const V rv = r[i];
    p[i] = rv + gg * p[i];
    for (int k = lo; k <= hi; k++) {
      const R om = VT<V>::cast(ms->omegas[k]), ga = VT<V>::cast(ms->gammas[k]), ze = VT<V>::cast(ms->zeta_iii[k]);
      V* o = out + k * stride;
      V* f = sf + k * stride;
      const V fv = f[i];
      o[i] = o[i] - om * fv;
      f[i] = ga * fv + ze * rv;
    }
  }
}

// :178-180, :230-275
__global__ void k_ms_converge(MsState* ms) {
  if (ms->done) return;
  ms_converge_step(ms);
}

template <class V>
__global__ void k_fill_shifts(V* sf, const V* in, size_t n, size_t stride, int nq) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    V v = in[i];
    for (int k = 0; k < nq; k++) sf[k * stride + i] = v;
  }
}

inline unsigned vec_grid(size_t n) {
  size_t b = (n + kThreads - 1) / kThreads;
  if (b > device_sms() * 8) b = device_sms() * 8;
  return (unsigned)(b ? b : 1);
}
}  // namespace

int ms_prepare_state(thr_ctx* c, MsState* h, int ndiagq, const double* aden, const double* anum, float res,
                     int maxcg) {
  if (ndiagq < 1 || ndiagq > kMaxShift) return THR_ERR_BADSHAPE;
  memset(h, 0, sizeof(MsState));
  // correction = |anum/aden| / geometric mean (:87-88)
  double slog = 0.0;
  for (int k = 0; k < ndiagq; k++) {
    h->correction[k] = std::fabs(anum[k] / aden[k]);
    slog += std::log(h->correction[k]);
  }
  const double gm = std::exp(slog / ndiagq);
  for (int k = 0; k < ndiagq; k++) {
    h->correction[k] = h->correction[k] / gm;
    h->flags[k] = 1;
    h->zeta_i[k] = 1.0;
    h->zeta_ii[k] = 1.0;
    h->gammas[k] = 0.0;
    h->aden[k] = aden[k];
  }
  h->omega = 1.0;
  h->gammag = 0.0;
  h->alpha = 0.0;
  h->ndiagq = ndiagq;
  h->lo = 0;
  h->hi = ndiagq - 1;
  h->maxcg = maxcg;
  h->res = res;
  h->done = (maxcg <= 0);
  (void)c;
  return THR_OK;
}

// Multishift solve on device vectors.  in: the source (precision V);
// out/sf: ndiagq shift fields each `stride` elements; r, p, h, s: work.
template <class V>
int multishift_dev(thr_ctx* c, const V* u_dummy, const V* in, V* out, V* sf, V* r, V* p, V* hv, V* s,
                   int ndiagq, const double* aden, const double* anum, float res, float am, int imass, int maxcg,
                   int* cg_return, int* cg_returns) {
  (void)u_dummy;
  const size_t n = c->n4();
  const size_t stride = n;
  MsState* ms = reinterpret_cast<MsState*>(c->dscal);
  MsState* h = reinterpret_cast<MsState*>(c->hscal);
  THR_TRY(ms_prepare_state(c, h, ndiagq, aden, anum, res, maxcg));
  THR_CUDA(cudaMemcpyAsync(ms, h, sizeof(MsState), cudaMemcpyHostToDevice, c->st));
  THR_CUDA(cudaMemcpyAsync(r, in, n * sizeof(V), cudaMemcpyDeviceToDevice, c->st));
  THR_CUDA(cudaMemcpyAsync(p, in, n * sizeof(V), cudaMemcpyDeviceToDevice, c->st));
  const unsigned gb = vec_grid(n);
  k_norm2<V><<<gb, kThreads, 0, c->st>>>(nullptr, r, n, c->partials);
  k_ms_init<<<1, 256, 0, c->st>>>(ms, c->partials, gb);
  THR_CUDA(cudaMemsetAsync(out, 0, (size_t)ndiagq * stride * sizeof(V), c->st));
  k_fill_shifts<V><<<gb, kThreads, 0, c->st>>>(sf, in, n, stride, ndiagq);
  const bool sp = sizeof(V) == sizeof(float2);
  const void* u = sp ? (const void*)c->u32 : (const void*)c->u64;
  const int chunk = 8;
  int it_host = 0;
  const double lb = sp ? sizeof(float2) : sizeof(double2);
  const double b_m = 2.0 * n * sizeof(V) + 3.0 * c->g.v3 * lb;
  const size_t prof_first = c->prof_kind.size();
  for (;;) {
    for (int k = 0; k < chunk; k++) {
      const long long tag = it_host + k;
      int pe = c->prof_begin(thr_ctx::P_DSLASH, b_m, tag);
      THR_TRY(launch_dslash_guarded<V>(c, false, hv, p, (const V*)u, am, imass, &ms->done));
      c->prof_end(pe);
      pe = c->prof_begin(thr_ctx::P_DSLASH, b_m, tag);
      THR_TRY(launch_dslash_guarded<V>(c, true, s, hv, (const V*)u, am, imass, &ms->done));
      c->prof_end(pe);
      k_redot<V><<<gb, kThreads, 0, c->st>>>(ms, p, s, n, c->partials);
      k_ms_alpha<<<1, 256, 0, c->st>>>(ms, c->partials, gb);
      k_ms_rupdate<V><<<gb, kThreads, 0, c->st>>>(ms, r, s, n, c->partials);
      k_ms_lambda<<<1, 256, 0, c->st>>>(ms, c->partials, gb);
      pe = c->prof_begin(thr_ctx::P_SHIFTUPD, 0.0, tag);
      k_ms_pshift<V><<<gb, kThreads, 0, c->st>>>(ms, p, r, out, sf, n, stride);
      c->prof_end(pe);
      k_ms_converge<<<1, 1, 0, c->st>>>(ms);
    }
    it_host += chunk;
    THR_CUDA(cudaMemcpyAsync(h, ms, sizeof(MsState), cudaMemcpyDeviceToHost, c->st));
    THR_CUDA(cudaStreamSynchronize(c->st));
    if (h->done) break;
    if (it_host > maxcg + 2 * chunk) return THR_ERR_CUDA;  // the device state stopped advancing
  }
  if (c->prof_on) {
    // shift update = r, p read + p write + (out, sf) read + write per active shift; the
    // active count of one iteration is not recorded, so each sampled launch gets the mean
    c->prof_trim(prof_first, h->it);
    const double per = h->it > 0 ? (3.0 + 4.0 * h->active_sum / h->it) * n * sizeof(V) : 0.0;
    for (size_t i = prof_first; i < c->prof_kind.size(); i++)
      if (c->prof_kind[i] == thr_ctx::P_SHIFTUPD) c->prof_bytes[i] = per;
    c->prof_work[thr_ctx::P_DSLASH] += 2.0 * h->it;
    c->prof_work[thr_ctx::P_SHIFTUPD] += h->it;
  }
  if (cg_return) *cg_return = h->it;
  if (cg_returns)
    for (int k = 0; k < ndiagq; k++) cg_returns[k] = h->cg_returns[k];
  return h->status ? h->status : THR_OK;
}

template int multishift_dev<double2>(thr_ctx*, const double2*, const double2*, double2*, double2*, double2*, double2*,
                                     double2*, double2*, int, const double*, const double*, float, float, int, int,
                                     int*, int*);
template int multishift_dev<float2>(thr_ctx*, const float2*, const float2*, float2*, float2*, float2*, float2*,
                                    float2*, float2*, int, const double*, const double*, float, float, int, int, int*,
                                    int*);

}  // namespace thr
