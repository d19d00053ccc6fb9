// bcg.cu -- batched congrad: many right-hand sides, or many independent
// lattices of uneven sizes, solved together (measurement solves,
// measure_module.F90:9-140, as used by measure_shamir/meson/fermion).
//
// Every operation of an iteration is one launch for the whole batch: the
// stencil walks the work blocks of all entries in one persistent grid, the
// vector kernels take the entry from blockIdx.y, and each entry keeps its
// own CG scalars in device memory (converged entries are skipped).
//
// Precision: FP64 is congrad itself (measure_module.F90:56-121) on every
// entry: one CG from r = b - A x0, stopped by the recursive residual on
// congrad's rule |r|^2 < 4*V*Ls*res^2 and never restarted, so the iteration
// counts are the reference's (the solution is accumulated as x0 + e, which
// differs from x += alpha p by rounding only).  The mixed modes keep x and
// the true residual in FP64 and solve each correction in low precision (FP32
// vectors, or BF16 storage of the stencil operands with FP32 arithmetic) to a
// relative 1e-5 / 1e-2, then recompute the FP64 true residual (defect
// correction) until every entry meets the rule on it.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "batch.h"
#include "bcg.h"
#include "ctx.h"
#include "thr_reduce.cuh"

namespace thr {

BatchTable::~BatchTable() { cudaFree(dev); }

int BatchTable::build(const std::vector<Geom>& geoms, bool shared_links, cudaStream_t st) {
  host.clear();
  nent = (int)geoms.size();
  total_blocks = 0;
  total_elems = 0;
  total_links = 0;
  for (const Geom& g : geoms) {
    if (g.ls < 1 || g.ls > 256) return THR_ERR_BADSHAPE;
    BatchEntry e{};
    e.g = g;
    e.off = total_elems;
    e.uoff = shared_links ? 0 : total_links;
    e.spb = std::max(1, 256 / g.ls);
    e.nblk = (g.v3 + e.spb - 1) / e.spb;
    e.blk0 = total_blocks;
    total_blocks += e.nblk;
    total_elems += g.v5 * 4;
    if (!shared_links || host.empty()) total_links += (long long)g.v3 * 3;
    host.push_back(e);
  }
  cudaFree(dev);
  dev = nullptr;
  if (cudaMalloc(&dev, sizeof(BatchEntry) * std::max(1, nent)) != cudaSuccess) return THR_ERR_NOMEM;
  if (cudaMemcpyAsync(dev, host.data(), sizeof(BatchEntry) * nent, cudaMemcpyHostToDevice, st) != cudaSuccess)
    return THR_ERR_CUDA;
  return THR_OK;
}

namespace {
constexpr int kT = 256;
constexpr int kGX = 64;  // blocks per entry in the vector kernels

template <class V> struct Pr;
template <> struct Pr<double2> {
  using R = double;
  static __device__ __forceinline__ double2 ld(const double2* p, size_t i) { return p[i]; }
  static __device__ __forceinline__ void st(double2* p, size_t i, double2 v) { p[i] = v; }
};
template <> struct Pr<float2> {
  using R = float;
  static __device__ __forceinline__ float2 ld(const float2* p, size_t i) { return p[i]; }
  static __device__ __forceinline__ void st(float2* p, size_t i, float2 v) { p[i] = v; }
};
template <> struct Pr<__nv_bfloat162> {
  using R = float;
  static __device__ __forceinline__ float2 ld(const __nv_bfloat162* p, size_t i) { return __bfloat1622float2(p[i]); }
  static __device__ __forceinline__ void st(__nv_bfloat162* p, size_t i, float2 v) { p[i] = __float22bfloat162_rn(v); }
};

// value in the arithmetic type of storage VS (double2 for FP64, float2 otherwise)
template <class VS> struct StC { using T = float2; };
template <> struct StC<double2> { using T = double2; };
template <class VS, class VA>
__device__ __forceinline__ typename StC<VS>::T make_float2_or_double2(VA v) {
  typename StC<VS>::T t;
  t.x = v.x;
  t.y = v.y;
  return t;
}

__device__ __forceinline__ void entry_range(const BatchEntry* tab, int e, size_t& off, size_t& n) {
  off = (size_t)tab[e].off;
  n = (size_t)tab[e].g.v5 * 4;
}

// sum of this entry's partials (one warp per entry, lanes stride, fixed order)
__device__ __forceinline__ double warp_entry_sum(const double* partials, int first, int count) {
  double v = 0.0;
  for (int i = threadIdx.x; i < count; i += 32) v += partials[first + i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return __shfl_sync(0xffffffffu, v, 0);
}

// R = B - T with |R|^2 partials (outer step, FP64)
__global__ void k_outer_res(const BatchEntry* tab, const BcgState* stt, const double2* B, const double2* T,
                            double2* R, double* partials) {
  const int e = blockIdx.y;
  double acc = 0.0;
  if (!stt[e].done_outer) {
    size_t off, n;
    entry_range(tab, e, off, n);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
      const double2 v = B[off + i] - T[off + i];
      R[off + i] = v;
      acc += v.x * v.x + v.y * v.y;
    }
  }
  block_write_partial(acc, partials + (size_t)e * gridDim.x);
}

__global__ void k_outer_check(BcgState* stt, int* skip, const double* partials, int gx, float tol_rel, int first) {
  const int e = blockIdx.x;
  const double r2 = warp_entry_sum(partials, e * gx, gx);
  if (threadIdx.x != 0) return;
  BcgState& s = stt[e];
  if (s.done_outer) return;
  s.r2_true = r2;
  if (!first) s.outer += 1;
  if (!(r2 == r2)) s.status = THR_ERR_NAN;
  if (r2 < s.resid || s.status || s.iters >= s.cap) s.done_outer = 1;
  else s.rounds += 1;  // a correction solve follows
  // FP64: the correction CG stops on congrad's own rule (|r|^2 < resid);
  // mixed: a relative reduction, never tighter than the rule needs
  s.target = tol_rel == 0.0f ? s.resid : fmax((double)tol_rel * (double)tol_rel * r2, 0.25 * s.resid);
  skip[e] = s.done_outer;
}

// r = R (low precision), p = r, e = 0, partials |r|^2
template <class VS, class VA>
__global__ void k_inner_init(const BatchEntry* tab, const BcgState* stt, const double2* R, VA* r, VS* p, VA* ev,
                             double* partials) {
  const int e = blockIdx.y;
  double acc = 0.0;
  if (!stt[e].done_outer) {
    size_t off, n;
    entry_range(tab, e, off, n);
    using RA = typename Pr<VA>::R;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
      const double2 v = R[off + i];
      VA rv;
      rv.x = (RA)v.x;
      rv.y = (RA)v.y;
      r[off + i] = rv;
      Pr<VS>::st(p, off + i, make_float2_or_double2<VS>(rv));
      VA z;
      z.x = RA(0);
      z.y = RA(0);
      ev[off + i] = z;
      acc += (double)rv.x * (double)rv.x + (double)rv.y * (double)rv.y;
    }
  }
  block_write_partial(acc, partials + (size_t)e * gridDim.x);
}

__global__ void k_inner_start(BcgState* stt, int* skip, const double* partials, int gx) {
  const int e = blockIdx.x;
  const double rr = warp_entry_sum(partials, e * gx, gx);
  if (threadIdx.x != 0) return;
  BcgState& s = stt[e];
  s.rr = rr;
  s.inner_it = 0;
  s.done_at = -1;  // no step of this inner solve has run
  s.done_inner = s.done_outer || !(rr > s.target);
  skip[e] = s.done_inner;
}

// pq from the stencil epilogue partials of the entry's work blocks; alpha = rr / pq
__global__ void k_alpha(const BatchEntry* tab, BcgState* stt, const double* partials) {
  const int e = blockIdx.x;
  if (stt[e].done_inner) return;
  const double pq = warp_entry_sum(partials, tab[e].blk0, tab[e].nblk);
  if (threadIdx.x == 0) stt[e].alpha = stt[e].rr / pq;
}

// measure_module.F90:102-110 with |r|^2 from the partials of the fused M^dagger stencil
// (r -= alpha M^dagger M p in its epilogue, one partial per work block of the entry)
__global__ void k_beta(const BatchEntry* tab, BcgState* stt, int* skip, const double* partials, int inner_cap,
                       int step) {
  const int e = blockIdx.x;
  if (stt[e].done_inner) return;
  const double rn = warp_entry_sum(partials, tab[e].blk0, tab[e].nblk);
  if (threadIdx.x != 0) return;
  BcgState& s = stt[e];
  s.beta = rn / s.rr;
  s.rr = rn;
  s.iters += 1;
  s.inner_it += 1;
  if (!(rn == rn)) {
    s.status = THR_ERR_NAN;
    s.done_outer = 1;
  }
  if (!(rn > s.target) || s.inner_it >= inner_cap || s.iters >= s.cap || s.status) {
    s.done_inner = 1;
    s.done_at = step;
  }
  skip[e] = s.done_inner;
}

// e += alpha p (:91); p = r + beta p (:110) -- one pass, the old p read once.  An entry
// whose solve ended at this step (done_at) still takes its last e update, not the p update.
template <class VS, class VA>
__global__ void k_xp(const BatchEntry* tab, const BcgState* stt, VA* ev, VS* p, const VA* r, int step) {
  const int e = blockIdx.y;
  const bool last = stt[e].done_inner;
  if (last && stt[e].done_at != step) return;
  size_t off, n;
  entry_range(tab, e, off, n);
  using RA = typename Pr<VA>::R;
  const RA a = (RA)stt[e].alpha, b = (RA)stt[e].beta;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const auto pv = Pr<VS>::ld(p, off + i);
    VA x = ev[off + i];
    x.x += a * (RA)pv.x;
    x.y += a * (RA)pv.y;
    ev[off + i] = x;
    if (!last) {
      const VA rv = r[off + i];
      VA v;
      v.x = rv.x + b * (RA)pv.x;
      v.y = rv.y + b * (RA)pv.y;
      Pr<VS>::st(p, off + i, make_float2_or_double2<VS>(v));
    }
  }
}

// X += e (FP64)
template <class VA>
__global__ void k_accumulate(const BatchEntry* tab, const BcgState* stt, double2* X, const VA* ev) {
  const int e = blockIdx.y;
  if (stt[e].done_outer) return;
  size_t off, n;
  entry_range(tab, e, off, n);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const VA v = ev[off + i];
    X[off + i] = X[off + i] + make_double2((double)v.x, (double)v.y);
  }
}

__global__ void k_reopen(BcgState* stt, int* skip, int nent) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < nent) skip[e] = stt[e].done_outer;
}

// FP64 (congrad): the entry is finished when its CG met the rule on the
// recursive residual; one that ran into the iteration cap stays open (MAXITER)
__global__ void k_close_fp64(BcgState* stt, int nent) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nent) return;
  BcgState& s = stt[e];
  if (!s.done_outer && !s.status && s.rr < s.resid) s.done_outer = 1;
}
}  // namespace

// FP64 operator T = M^dagger M X on the batch
static int batch_mdagm(BcgRun& br, const double2* X, double2* T, double2* H) {
  THR_TRY(launch_dslash_batch<double2>(*br.tab, br.kernel, false, H, X, br.u64, br.am, br.imass, br.am3, br.st,
                                       br.skip, nullptr, nullptr, br.grid));
  return launch_dslash_batch<double2>(*br.tab, br.kernel, true, T, H, br.u64, br.am, br.imass, br.am3, br.st, br.skip,
                                      nullptr, nullptr, br.grid);
}

template <class VS, class VA>
static int bcg_inner(BcgRun& br, VA* r, VS* p, VS* h, VS* q, VA* ev, float tol, int inner_cap) {
  const BatchTable& tab = *br.tab;
  const dim3 vg(kGX, tab.nent);
  const typename Sto<VS>::C* u = (const typename Sto<VS>::C*)br.ulow;
  if (sizeof(VS) == sizeof(double2)) u = (const typename Sto<VS>::C*)(const void*)br.u64;
  k_inner_init<VS, VA><<<vg, kT, 0, br.st>>>(tab.dev, br.state, br.R, r, p, ev, br.partials);
  k_inner_start<<<tab.nent, 32, 0, br.st>>>(br.state, br.skip, br.partials, kGX);
  const int chunk = 16;
  std::vector<BcgState> h_state(tab.nent);
  // per step: h = M p with |h|^2 = |M p|^2 (the reference's alphad, :70); alpha; r -= alpha
  // M^dagger h with |r|^2 in the M^dagger epilogue (q = M^dagger M p never stored); beta;
  // e += alpha p and p = r + beta p in one pass.  r is held in the stencil's arithmetic type.
  static_assert(sizeof(BcgState) % sizeof(double) == 0, "BcgState scalars are addressed with a stride");
  const int stride = (int)(sizeof(BcgState) / sizeof(double));
  const double* alpha0 = &br.state[0].alpha;
  using C = typename Sto<VS>::C;
  static_assert(sizeof(C) == sizeof(VA), "r is held in the stencil's arithmetic type");
  (void)q;
  for (int it = 0; it < inner_cap + chunk; it += chunk) {
    for (int k = 0; k < chunk; k++) {
      const int step = it + k;
      THR_TRY(launch_dslash_batch_fused<VS>(tab, br.kernel, false, 2, h, p, u, br.am, br.imass, br.am3, br.st,
                                            br.skip, nullptr, nullptr, 0, br.partials, br.grid));
      k_alpha<<<tab.nent, 32, 0, br.st>>>(tab.dev, br.state, br.partials);
      THR_TRY(launch_dslash_batch_fused<VS>(tab, br.kernel, true, 4, nullptr, h, u, br.am, br.imass, br.am3, br.st,
                                            br.skip, reinterpret_cast<C*>(r), alpha0, stride, br.partials, br.grid));
      k_beta<<<tab.nent, 32, 0, br.st>>>(tab.dev, br.state, br.skip, br.partials, inner_cap, step);
      k_xp<VS, VA><<<vg, kT, 0, br.st>>>(tab.dev, br.state, ev, p, r, step);
      br.launches += 5;
    }
    THR_CUDA(cudaMemcpyAsync(h_state.data(), br.state, sizeof(BcgState) * tab.nent, cudaMemcpyDeviceToHost, br.st));
    THR_CUDA(cudaStreamSynchronize(br.st));
    bool all = true;
    for (auto& s : h_state) all = all && s.done_inner;
    if (all) break;
  }
  (void)tol;
  return THR_OK;
}

int bcg_solve(BcgRun& br, int precision, float res, int max_outer, int* iters, int* outer) {
  const BatchTable& tab = *br.tab;
  const int ne = tab.nent;
  std::vector<BcgState> h(ne);
  for (int e = 0; e < ne; e++) {
    const Geom& g = tab.host[e].g;
    const int ivol = 4 * g.lx * g.ly * g.lt * g.ls;
    const float resid = ((float)ivol * res) * res;  // measure_module.F90:41
    h[e] = BcgState{};
    h[e].resid = (double)resid;
    h[e].cap = g.ls * g.v3;  // niterc, params.F90:57
  }
  THR_CUDA(cudaMemcpyAsync(br.state, h.data(), sizeof(BcgState) * ne, cudaMemcpyHostToDevice, br.st));
  THR_CUDA(cudaMemsetAsync(br.skip, 0, sizeof(int) * ne, br.st));
  const dim3 vg(kGX, ne);
  const float tol = precision == THR_FP64 ? 0.0f : (precision == THR_MIXED_BF16 ? 1e-2f : 1e-5f);
  const int inner_cap = 1 << 30;
  int rounds = 0;
  for (int outer_it = 0; outer_it < max_outer; outer_it++) {
    // true residual in FP64
    k_reopen<<<(ne + 127) / 128, 128, 0, br.st>>>(br.state, br.skip, ne);
    THR_TRY(batch_mdagm(br, br.X, br.T, br.H));
    k_outer_res<<<vg, kT, 0, br.st>>>(tab.dev, br.state, br.B, br.T, br.R, br.partials);
    k_outer_check<<<ne, 32, 0, br.st>>>(br.state, br.skip, br.partials, kGX, tol, outer_it == 0);
    br.launches += 4;
    THR_CUDA(cudaMemcpyAsync(h.data(), br.state, sizeof(BcgState) * ne, cudaMemcpyDeviceToHost, br.st));
    THR_CUDA(cudaStreamSynchronize(br.st));
    bool all = true;
    for (auto& s : h) all = all && s.done_outer;
    if (all) break;
    rounds++;
    // correction solve
    if (precision == THR_FP64) {
      THR_TRY(bcg_inner<double2, double2>(br, (double2*)br.r, (double2*)br.p, (double2*)br.h, (double2*)br.q,
                                          (double2*)br.e, tol, inner_cap));
      k_accumulate<double2><<<vg, kT, 0, br.st>>>(tab.dev, br.state, br.X, (const double2*)br.e);
      k_close_fp64<<<(ne + 127) / 128, 128, 0, br.st>>>(br.state, ne);
      br.launches += 2;
      break;  // congrad never restarts
    } else if (precision == THR_MIXED_BF16) {
      THR_TRY(bcg_inner<__nv_bfloat162, float2>(br, (float2*)br.r, (__nv_bfloat162*)br.p, (__nv_bfloat162*)br.h,
                                                (__nv_bfloat162*)br.q, (float2*)br.e, tol, inner_cap));
      k_accumulate<float2><<<vg, kT, 0, br.st>>>(tab.dev, br.state, br.X, (const float2*)br.e);
    } else {
      THR_TRY(bcg_inner<float2, float2>(br, (float2*)br.r, (float2*)br.p, (float2*)br.h, (float2*)br.q, (float2*)br.e,
                                        tol, inner_cap));
      k_accumulate<float2><<<vg, kT, 0, br.st>>>(tab.dev, br.state, br.X, (const float2*)br.e);
    }
    br.launches += 1;
  }
  THR_CUDA(cudaMemcpyAsync(h.data(), br.state, sizeof(BcgState) * ne, cudaMemcpyDeviceToHost, br.st));
  THR_CUDA(cudaStreamSynchronize(br.st));
  int rc = THR_OK;
  for (int e = 0; e < ne; e++) {
    // CG steps plus one per FP64 residual that started a correction (the
    // reference counts its initial-residual pass as an iteration too: in FP64
    // that pass is always one, itercg = 1 when the guess already meets the rule)
    if (iters) iters[e] = h[e].iters + (precision == THR_FP64 ? 1 : h[e].rounds);
    if (h[e].status) rc = h[e].status;
    else if (!h[e].done_outer && rc == THR_OK) rc = THR_ERR_MAXITER;
  }
  if (outer) *outer = rounds;
  return rc;
}

}  // namespace thr
