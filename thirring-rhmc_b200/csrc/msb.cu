// msb.cu -- multishift CG with batched shift updates.
//
// Same recurrences as multishift_module.F90:13-284 (and :289-534 for FP32
// vectors), reorganised for HBM traffic.  The reference updates every
// active shift field in every iteration (4 passes per shift per iteration,
// :155-176).  Here each iteration only writes its new residual r_k into a
// ring of kBatch+1 fields and records the iteration's per-shift
// coefficients (omegas, gammas, zeta_iii and the active window); every
// kBatch iterations the recorded updates
//     for j in batch:  out -= om_j * sf ;  sf = ga_j * sf + ze_j * r_j
// are folded per shift into one affine map of the batch's start values
// (k_flush_coef) and applied in one pass over the shift fields (k_flush).
// The algebra is that of the per-iteration form; only the rounding order
// differs.  Traffic per iteration drops from (3 + 4 n_active) to about
// (1 + 4 n_active / kBatch) fields.  In addition alpha = Re<p, M^dagger M p>
// is accumulated in the epilogue of the M^dagger stencil, so s is not re-read.
#include <cmath>
#include <cstring>

#include "ctx.h"
#include "ms.h"
#include "solver.h"
#include "thr_reduce.cuh"

namespace thr {

namespace {
constexpr int kThreads = 256;

template <class V> struct W;
template <> struct W<double2> {
  using R = double;
  static __device__ __forceinline__ double abs2(double2 a) { return a.x * a.x + a.y * a.y; }
  static __device__ __forceinline__ double cast(double v) { return v; }
};
template <> struct W<float2> {
  using R = float;
  static __device__ __forceinline__ double abs2(float2 a) { return (double)(a.x * a.x + a.y * a.y); }
  static __device__ __forceinline__ float cast(double v) { return (float)v; }
};

template <class V>
__global__ void k_norm2(const V* a, size_t n, double* partials) {
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    acc += W<V>::abs2(a[i]);
  block_write_partial(acc, partials);
}
__global__ void k_init(MsState* ms, MsHist* hist, const double* partials, int np) {
  const double d = block_sum_partials(partials, np);
  if (threadIdx.x == 0) {
    ms->delta = d;
    hist->nsteps = 0;
  }
}

// :104, :118-135, recording the step's omegas / zeta_iii / window
__global__ void k_alpha(MsState* ms, MsHist* hist, const double* partials, int np) {
  if (ms->done) return;
  const double alpha = block_sum_partials(partials, np);
  if (threadIdx.x == 0) {
    ms_alpha_scalar(ms, alpha);
    hist->lo[hist->nsteps] = ms->lo;
    hist->hi[hist->nsteps] = ms->hi;
  }
  __syncthreads();
  const int k = ms->lo + threadIdx.x;
  if (k <= ms->hi) {
    ms_alpha_shift(ms, k);
    hist->om[hist->nsteps][k] = ms->omegas[k];
    hist->ze[hist->nsteps][k] = ms->zeta_iii[k];
  }
}

// r_new = r_old + omega*s (:137), lambda partials (:138)
template <class V>
__global__ void k_rupdate(const MsState* ms, V* rnew, const V* rold, const V* s, size_t n, double* partials) {
  if (ms->done) return;
  using R = typename W<V>::R;
  const R om = W<V>::cast(ms->omega);
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const V v = rold[i] + om * s[i];
    rnew[i] = v;
    acc += W<V>::abs2(v);
  }
  block_write_partial(acc, partials);
}

// :143, :148-150, recording gammas; closes the step's record
__global__ void k_lambda(MsState* ms, MsHist* hist, const double* partials, int np) {
  if (ms->done) return;
  const double lambda = block_sum_partials(partials, np);
  if (threadIdx.x == 0) ms_lambda_scalar(ms, lambda);
  __syncthreads();
  const int k = ms->lo + threadIdx.x;
  if (k <= ms->hi) {
    ms_lambda_shift(ms, k);
    hist->ga[hist->nsteps][k] = ms->gammas[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) hist->nsteps += 1;
}

// p = r + gammag*p (:145)
template <class V>
__global__ void k_pupdate(const MsState* ms, V* p, const V* r, size_t n) {
  if (ms->done) return;
  using R = typename W<V>::R;
  const R gg = W<V>::cast(ms->gammag);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    p[i] = r[i] + gg * p[i];
}

__global__ void k_converge(MsState* ms) {
  if (ms->done) return;
  ms_converge_step(ms);
}

// Fold each shift's recorded steps (:155-176 once per step) into one affine map
// of the batch's start values: with f = sf, o = out,
//   step j (if shift k is in that step's window):  o -= om_j f ;  f = ga_j f + ze_j r_j
// gives  f_end = A f_0 + sum_i B_i r_i   and   o_end = o_0 - P f_0 - sum_i Q_i r_i.
// One thread per shift; the map is exact algebra, only the rounding differs.
__global__ void k_flush_coef(MsState* ms, const MsHist* hist, MsCoef* cf) {
  const int ns = hist->nsteps;
  const int k = threadIdx.x;
  if (k == 0) {
    int lo_u = kMaxShift, hi_u = -1;
    for (int j = 0; j < ns; j++) {
      lo_u = min(lo_u, hist->lo[j]);
      hi_u = max(hi_u, hist->hi[j]);
    }
    cf->ns = ns;
    cf->lo = lo_u;
    cf->hi = hi_u;
    if (ns > 0) ms->flush_fields += (double)(ns + 4 * (hi_u - lo_u + 1));
  }
  if (k >= kMaxShift) return;
  double A = 1.0, P = 0.0, B[kBatch], Q[kBatch];
#pragma unroll
  for (int i = 0; i < kBatch; i++) B[i] = Q[i] = 0.0;
#pragma unroll
  for (int j = 0; j < kBatch; j++) {
    if (j < ns && k >= hist->lo[j] && k <= hist->hi[j]) {
      const double om = hist->om[j][k], ga = hist->ga[j][k], ze = hist->ze[j][k];
      P += om * A;
#pragma unroll
      for (int i = 0; i < kBatch; i++)
        if (i < j) Q[i] += om * B[i];
      A = ga * A;
#pragma unroll
      for (int i = 0; i < kBatch; i++)
        if (i < j) B[i] = ga * B[i];
      B[j] = ze;
    }
  }
  cf->A[k] = A;
  cf->P[k] = P;
#pragma unroll
  for (int i = 0; i < kBatch; i++) {
    cf->B[k][i] = B[i];
    cf->Q[k][i] = Q[i];
  }
}

// apply the folded maps to every shift field of the batch's window
template <class V>
__global__ void __launch_bounds__(kThreads) k_flush(const MsCoef* cf, V* __restrict__ out, V* __restrict__ sf,
                                                   const V* __restrict__ ring, int base, int ring_len, size_t n,
                                                   size_t stride) {
  using R = typename W<V>::R;
  const int ns = cf->ns;
  if (ns == 0) return;
  const int lo = cf->lo, hi = cf->hi;
  __shared__ R s_A[kMaxShift], s_P[kMaxShift], s_B[kMaxShift][kBatch], s_Q[kMaxShift][kBatch];
  for (int t = threadIdx.x; t < kMaxShift * kBatch; t += blockDim.x) {
    const int k = t / kBatch, i = t % kBatch;
    s_B[k][i] = (R)cf->B[k][i];
    s_Q[k][i] = (R)cf->Q[k][i];
    if (i == 0) {
      s_A[k] = (R)cf->A[k];
      s_P[k] = (R)cf->P[k];
    }
  }
  __syncthreads();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    V rj[kBatch];
#pragma unroll
    for (int j = 0; j < kBatch; j++)
      if (j < ns) rj[j] = ring[(size_t)((base + 1 + j) % ring_len) * n + i];
    for (int k = lo; k <= hi; k++) {
      const V f0 = sf[k * stride + i];
      const V o0 = out[k * stride + i];
      V f = s_A[k] * f0;
      V o = o0 - s_P[k] * f0;
#pragma unroll
      for (int j = 0; j < kBatch; j++) {
        if (j < ns) {
          f = f + s_B[k][j] * rj[j];
          o = o - s_Q[k][j] * rj[j];
        }
      }
      sf[k * stride + i] = f;
      out[k * stride + i] = o;
    }
  }
}
__global__ void k_reset(MsHist* hist) { hist->nsteps = 0; }

template <class V>
__global__ void k_fill(V* sf, const V* in, size_t n, size_t stride, int nq) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const V v = in[i];
    for (int k = 0; k < nq; k++) sf[k * stride + i] = v;
  }
}

inline unsigned vec_grid(size_t n) {
  size_t b = (n + kThreads - 1) / kThreads;
  if (b > 148 * 8) b = 148 * 8;
  return (unsigned)(b ? b : 1);
}
}  // namespace

template <class V>
int multishift_batched_dev(thr_ctx* c, const V* in, V* out, V* sf, V* ring, V* p, V* hv, V* s, int ndiagq,
                           const double* aden, const double* anum, float res, float am, int imass, int maxcg,
                           int* cg_return, int* cg_returns) {
  const size_t n = c->n4();
  const size_t stride = n;
  const int ring_len = kBatch + 1;
  MsState* ms = reinterpret_cast<MsState*>(c->dscal);
  MsState* h = reinterpret_cast<MsState*>(c->hscal);
  void* hv_;
  THR_TRY(c->buffer(thr_ctx::B_HIST, sizeof(MsHist), &hv_));
  MsHist* hist = (MsHist*)hv_;
  void* cf_;
  THR_TRY(c->buffer(thr_ctx::B_COEF, sizeof(MsCoef), &cf_));
  MsCoef* cf = (MsCoef*)cf_;
  THR_TRY(ms_prepare_state(c, h, ndiagq, aden, anum, res, maxcg));
  THR_CUDA(cudaMemcpyAsync(ms, h, sizeof(MsState), cudaMemcpyHostToDevice, c->st));
  THR_CUDA(cudaMemcpyAsync(ring, in, n * sizeof(V), cudaMemcpyDeviceToDevice, c->st));  // r = input (slot 0)
  THR_CUDA(cudaMemcpyAsync(p, in, n * sizeof(V), cudaMemcpyDeviceToDevice, c->st));     // p = r
  const unsigned gb = vec_grid(n);
  k_norm2<V><<<gb, kThreads, 0, c->st>>>(ring, n, c->partials);
  k_init<<<1, kThreads, 0, c->st>>>(ms, hist, c->partials, gb);
  THR_CUDA(cudaMemsetAsync(out, 0, (size_t)ndiagq * stride * sizeof(V), c->st));
  k_fill<V><<<gb, kThreads, 0, c->st>>>(sf, in, n, stride, ndiagq);
  const bool sp = sizeof(V) == sizeof(float2);
  const V* u = sp ? (const V*)(const void*)c->u32 : (const V*)(const void*)c->u64;
  const unsigned gs = stencil_grid(c->g, c->p.kernel);
  // algorithmic bytes: M reads R, writes Phi, reads the links; M^dagger with the
  // fused <p, M^dagger M p> also reads p
  const double lb = sp ? sizeof(float2) : sizeof(double2);
  const double b_m = 2.0 * n * sizeof(V) + 3.0 * c->g.v3 * lb, b_md = b_m + (double)n * sizeof(V);
  const size_t prof_first = c->prof_kind.size();
  double flushed = 0.0;
  long long flushes = 0;
  long long k = 0;
  for (;;) {
    const long long base = k;
    for (int j = 0; j < kBatch; j++, k++) {
      V* rold = ring + (size_t)(k % ring_len) * n;
      V* rnew = ring + (size_t)((k + 1) % ring_len) * n;
      int pe = c->prof_begin(thr_ctx::P_DSLASH, b_m, k);
      THR_TRY(launch_dslash<V>(c->g, c->p.kernel, false, hv, p, (const typename Sto<V>::C*)u, am, imass, c->p.am3,
                               c->st, &ms->done));
      c->prof_end(pe);
      pe = c->prof_begin(thr_ctx::P_DSLASH_EPI, b_md, k);
      THR_TRY(launch_dslash_epi<V>(c->g, c->p.kernel, true, s, hv, (const typename Sto<V>::C*)u, am, imass,
                                   c->p.am3, c->st, &ms->done, p, c->partials));
      c->prof_end(pe);
      k_alpha<<<1, 1024, 0, c->st>>>(ms, hist, c->partials, gs);
      k_rupdate<V><<<gb, kThreads, 0, c->st>>>(ms, rnew, rold, s, n, c->partials);
      k_lambda<<<1, kThreads, 0, c->st>>>(ms, hist, c->partials, gb);
      k_pupdate<V><<<gb, kThreads, 0, c->st>>>(ms, p, rnew, n);
      k_converge<<<1, 1, 0, c->st>>>(ms);
    }
    int pe = c->prof_begin(thr_ctx::P_SHIFTUPD, 0.0, base);
    k_flush_coef<<<1, kMaxShift, 0, c->st>>>(ms, hist, cf);
    k_flush<V><<<gb, kThreads, 0, c->st>>>(cf, out, sf, ring, (int)(base % ring_len), ring_len, n, stride);
    c->prof_end(pe);
    k_reset<<<1, 1, 0, c->st>>>(hist);
    THR_CUDA(cudaMemcpyAsync(h, ms, sizeof(MsState), cudaMemcpyDeviceToHost, c->st));
    THR_CUDA(cudaStreamSynchronize(c->st));
    // flush traffic: each recorded step's residual read once, each shift field of the
    // batch's window read and written once (out and sf)
    c->prof_set_bytes(pe, (h->flush_fields - flushed) * n * sizeof(V));
    if (h->flush_fields > flushed) flushes++;
    flushed = h->flush_fields;
    if (h->done) break;
    if (k > (long long)maxcg + 2 * kBatch) return THR_ERR_CUDA;  // the device state stopped advancing
  }
  if (c->prof_on) {
    c->prof_trim(prof_first, h->it);  // launches after convergence skipped their work
    c->prof_work[thr_ctx::P_DSLASH] += h->it;
    c->prof_work[thr_ctx::P_DSLASH_EPI] += h->it;
    c->prof_work[thr_ctx::P_SHIFTUPD] += flushes;
  }
  if (cg_return) *cg_return = h->it;
  if (cg_returns)
    for (int q = 0; q < ndiagq; q++) cg_returns[q] = h->cg_returns[q];
  return h->status ? h->status : THR_OK;
}

template int multishift_batched_dev<double2>(thr_ctx*, const double2*, double2*, double2*, double2*, double2*,
                                             double2*, double2*, int, const double*, const double*, float, float, int,
                                             int, int*, int*);
template int multishift_batched_dev<float2>(thr_ctx*, const float2*, float2*, float2*, float2*, float2*, float2*,
                                            float2*, int, const double*, const double*, float, float, int, int, int*,
                                            int*);

}  // namespace thr
