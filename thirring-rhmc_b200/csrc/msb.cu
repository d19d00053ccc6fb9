// msb.cu -- multishift CG with batched shift updates.
//
// Same recurrences as multishift_module.F90:13-284 (and :289-534 for FP32
// vectors), reorganised for HBM traffic.  The reference updates every
// active shift field in every iteration (4 passes per shift per iteration,
// :155-176).  Here each iteration only writes its new residual r_k into a
// circular ring of 2 kBatch fields and records the iteration's per-shift
// coefficients (omegas, gammas, zeta_iii and the active window); every
// kBatch iterations (a batch, one half of the ring) the recorded updates
//     for j in batch:  out -= om_j * sf ;  sf = ga_j * sf + ze_j * r_j
// are folded per shift into one affine map of the batch's start values
// (k_flush_coef) and applied in one pass over the shift fields (k_flush).
// The algebra is that of the per-iteration form; only the rounding order
// differs.  Traffic per iteration drops from (3 + 4 n_active) to about
// (1 + 4 n_active / kBatch) fields.  A batch's flush runs on the context's
// low-priority side stream while the next batch iterates on the main stream
// (it reads the other half of the ring and the other of two histories), so
// the bandwidth-bound flush fills the time the latency-bound stencils and the
// one-block scalar kernels leave unused.  The search direction p enters the
// base recurrence only through h = M p, which is kept by h_new = M r + gammag h
// (p = r + gammag p and linearity), so p is never formed and the p update pass
// is gone; alpha = Re<p, M^dagger M p> (= |h|^2) is accumulated in the epilogue
// of the M stencil from the values it writes, so neither h nor s is re-read for it.
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
// hist: the two batch histories (both start empty)
__global__ void k_init(MsState* ms, MsHist* hist, const double* partials, int np) {
  const double d = block_sum_partials(partials, np);
  if (threadIdx.x == 0) {
    ms->delta = d;
    ms->switch_delta = ms->switch_rel2 * d;
    hist[0].nsteps = 0;
    hist[1].nsteps = 0;
  }
}

// The two scalar steps of an iteration, one block each.  The solver state is copied into
// shared memory at the start (one load per thread, issued with the partials' loads) and
// the step runs on the copy, so that its chain of dependent scalar accesses costs
// shared-memory latency instead of an L2 round trip each; the fields the step changes are
// written back at the end (not batches or flush_fields: the side stream's flush of the
// other ring half updates those meanwhile).  The arithmetic is ms_alpha_block's and
// ms_lambda_block's.
constexpr int kMsWords = (int)(sizeof(MsState) / sizeof(double));
static_assert(sizeof(MsState) % sizeof(double) == 0, "MsState is copied as doubles");
__device__ __forceinline__ void ms_stage(MsState* st, const MsState* ms) {
  double* dst = reinterpret_cast<double*>(st);
  const double* src = reinterpret_cast<const double*>(ms);
  for (int i = threadIdx.x; i < kMsWords; i += blockDim.x) dst[i] = src[i];
}

// :104, :118-135, recording the step's omegas / zeta_iii / window
__global__ void k_alpha(MsState* ms, MsHist* hist, const double* partials, int np) {
  pdl_wait();
  pdl_trigger();
  __shared__ MsState st;
  const int nsteps = hist->nsteps;
  ms_stage(&st, ms);
  const double alpha = block_sum_partials(partials, np);  // its barriers publish the copy
  if (st.done) return;
  ms_alpha_block(&st, hist, nsteps, alpha, threadIdx.x);
  __syncthreads();
  const int k = threadIdx.x;
  if (k == 0) {
    ms->it = st.it;
    ms->alpha = st.alpha;
    ms->omega_save = st.omega_save;
    ms->omega = st.omega;
  }
  if (k < kMaxShift) {
    ms->zeta_iii[k] = st.zeta_iii[k];
    ms->omegas[k] = st.omegas[k];
  }
}

// :143, :148-150, recording gammas; closes the step's record and ends the step
// (convergence test, window, delta: ms_lambda_block)
__global__ void k_lambda(MsState* ms, MsHist* hist, const double* partials, int np) {
  pdl_wait();
  pdl_trigger();
  __shared__ MsState st;
  __shared__ int s_lo, s_hi;
  const int nsteps = hist->nsteps;
  ms_stage(&st, ms);
  const double lambda = block_sum_partials(partials, np);
  if (st.done) return;
  ms_lambda_block(&st, hist, nsteps, lambda, threadIdx.x, &s_lo, &s_hi);
  __syncthreads();
  const int k = threadIdx.x;
  if (k == 0) {
    ms->lambda = st.lambda;
    ms->active_sum = st.active_sum;
    ms->gammag = st.gammag;
    ms->lo = st.lo;
    ms->hi = st.hi;
    ms->delta = st.delta;
    ms->status = st.status;
    ms->done = st.done;
  }
  if (k < kMaxShift) {
    ms->gammas[k] = st.gammas[k];
    ms->cg_returns[k] = st.cg_returns[k];
    ms->flags[k] = st.flags[k];
    ms->zeta_i[k] = st.zeta_i[k];
    ms->zeta_ii[k] = st.zeta_ii[k];
  }
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

// apply the folded maps to every shift field of the batch's window (the
// residual of the batch's step j is in ring slot (first + j) mod 2 kBatch).  One
// thread per element holds the batch's residuals in registers (kBatch values)
// and walks the window; the next shift's two fields are loaded while the
// current one is combined.
constexpr int kFlushThreads = 128;
constexpr int kFlushBlocks = 3;  // resident per SM at the register budget of kBatch residuals
// a ring value in the shift fields' complex type (exact widening)
__device__ __forceinline__ double2 widen(double2 v, double2) { return v; }
__device__ __forceinline__ double2 widen(float2 v, double2) { return make_double2((double)v.x, (double)v.y); }
__device__ __forceinline__ double2 widen(__nv_bfloat162 v, double2) {
  const float2 f = __bfloat1622float2(v);
  return make_double2((double)f.x, (double)f.y);
}
__device__ __forceinline__ float2 widen(float2 v, float2) { return v; }

template <class V, class VR = V>
__global__ void __launch_bounds__(kFlushThreads, kFlushBlocks)
    k_flush(const MsCoef* cf, V* __restrict__ out, V* __restrict__ sf, const VR* __restrict__ ring, size_t n,
            size_t stride, int first) {
  using R = typename W<V>::R;
  const int ns = cf->ns;
  if (ns == 0) return;
  const int lo = cf->lo, hi = cf->hi;  // lo > hi: no shift active in the batch
  if (lo > hi) return;
  // the maps of the window's shifts (the only rows read below)
  // B and Q of a (shift, step) side by side: one 16-byte (FP64) shared load per term of the FMA chains
  using R2 = typename Sto<V>::C;
  __shared__ R s_A[kMaxShift], s_P[kMaxShift];
  __shared__ R2 s_BQ[kMaxShift][kBatch];
  for (int t = threadIdx.x; t < (hi - lo + 1) * kBatch; t += blockDim.x) {
    const int k = lo + t / kBatch, i = t % kBatch;
    s_BQ[k][i] = mk((R)cf->B[k][i], (R)cf->Q[k][i]);
    if (i == 0) {
      s_A[k] = (R)cf->A[k];
      s_P[k] = (R)cf->P[k];
    }
  }
  __syncthreads();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    VR rj[kBatch];  // held in the ring's own type, widened where used
#pragma unroll
    for (int j = 0; j < kBatch; j++) {
      const int slot = first + j < 2 * kBatch ? first + j : first + j - 2 * kBatch;
      if (j < ns) rj[j] = ring[(size_t)slot * n + i];
    }
    V f0n = sf[lo * stride + i], o0n = out[lo * stride + i];
    for (int k = lo; k <= hi; k++) {
      const V f0 = f0n, o0 = o0n;
      if (k < hi) {
        f0n = sf[(k + 1) * stride + i];
        o0n = out[(k + 1) * stride + i];
      }
      V f = s_A[k] * f0;
      V o = o0 - s_P[k] * f0;
#pragma unroll
      for (int j = 0; j < kBatch; j++) {
        if (j < ns) {
          const R2 bq = s_BQ[k][j];
          const V r = widen(rj[j], V{});
          f = f + bq.x * r;
          o = o - bq.y * r;
        }
      }
      sf[k * stride + i] = f;
      out[k * stride + i] = o;
    }
  }
}
// short-lived blocks (at most kFlushPerThread elements per thread), so that a
// flush running beside the main chain interleaves with its kernels block by block
constexpr int kFlushPerThread = 4;
inline unsigned flush_grid(size_t n) {
  const size_t per = (size_t)kFlushThreads * kFlushPerThread;
  const size_t b = (n + per - 1) / per;
  return (unsigned)(b ? b : 1);
}
// close a batch
__global__ void k_reset(MsHist* hist, MsState* ms) {
  hist->nsteps = 0;
  ms->batches += 1;
}

// Loop control of the graph-driven solve: run another batch unless the solve is
// done.  max_batches bounds the loop whatever the device state holds (the
// recurrences stop at maxcg iterations; this is the backstop).
__global__ void k_loop_ctl(MsState* ms, cudaGraphConditionalHandle h) {
  unsigned more = 1u;
  if (ms->done) {
    more = 0u;
  } else if (ms->switch_delta > 0.0 && ms->delta < ms->switch_delta) {
    more = 0u;  // the FP64 phase of a mixed solve ends here (after this pair of batches)
  } else if (ms->batches >= ms->max_batches) {
    ms->status = THR_ERR_MAXITER;
    ms->done = 1;
    more = 0u;
  }
  cudaGraphSetConditional(h, more);
}

template <class V>
__global__ void k_fill(V* sf, const V* in, size_t n, size_t stride, int nq) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const V v = in[i];
    for (int k = 0; k < nq; k++) sf[k * stride + i] = v;
  }
}

inline unsigned vec_grid(size_t n) {
  size_t b = (n + kThreads - 1) / kThreads;
  if (b > device_sms() * 8) b = device_sms() * 8;
  return (unsigned)(b ? b : 1);
}
}  // namespace

namespace {
// flush of the batch recorded in hist (ring half `half`) on stream `on`; the
// shift fields are VO, the ring V
template <class V, class VO = V>
void enqueue_flush(thr_ctx* c, cudaStream_t on, MsState* ms, MsHist* hist, MsCoef* cf, VO* out, VO* sf, const V* ring,
                   int half, bool prof, long long tag, int* prof_flush) {
  const size_t n = c->n4();
  const int pe = prof ? c->prof_begin(thr_ctx::P_SHIFTUPD, 0.0, tag, on) : -1;
  k_flush_coef<<<1, kMaxShift, 0, on>>>(ms, hist, cf);
  k_flush<VO, V><<<flush_grid(n), kFlushThreads, 0, on>>>(cf, out, sf, ring, n, n, half * kBatch + 1);
  c->prof_end(pe, on);
  if (prof_flush) *prof_flush = pe;
  k_reset<<<1, 1, 0, on>>>(hist, ms);
}

// One batch of kBatch iterations on ring half `half` (stream order on `main`),
// recording into hist[half]; alongside it, on c->st2, the flush of the batch
// before (hist[1 - half], the other half).  Ring slots: iteration j of the batch
// reads r from slot half*kBatch + j and writes the new r to the next slot (mod
// 2 kBatch), so each half's batch starts from the other half's last residual.
// prof: sample kernel timings with events (stream-launched solves only).
template <class V, class VO = V>
int enqueue_batch(thr_ctx* c, MsState* ms, MsHist* hist, MsCoef* cf, VO* out, VO* sf, V* ring, V* p, V* hv, V* s,
                  float am, int imass, int half, long long k0, bool prof, int* prof_flush, cudaStream_t main) {
  const size_t n = c->n4();
  const unsigned gb = vec_grid(n / 4);
  const bool fp64 = sizeof(V) == sizeof(double2);
  const unsigned gs = stencil_parts(c->g, c->p.kernel, fp64);
  const typename Sto<V>::C* u =
      fp64 ? (const typename Sto<V>::C*)(const void*)c->u64 : (const typename Sto<V>::C*)(const void*)c->u32;
  const double lb = fp64 ? sizeof(double2) : sizeof(float2);
  const bool pdl = c->use_pdl && !prof;  // sampled launches keep their events between kernels
  // the previous batch's flush, forked onto the side stream (c->overlap_flush 0: in line;
  // also in line while kernel timings are sampled, so that each sampled duration is
  // that kernel's alone and not one shared with a concurrent flush)
  const bool fork = c->overlap_flush != 0 && !prof;
  if (fork) {
    THR_CUDA(cudaEventRecord(c->ev_fork[half], main));
    THR_CUDA(cudaStreamWaitEvent(c->st2, c->ev_fork[half], 0));
  }
  enqueue_flush<V, VO>(c, fork ? c->st2 : main, ms, hist + (1 - half), cf + (1 - half), out, sf, ring, 1 - half,
                       prof, k0 - kBatch, prof_flush);
  if (fork) THR_CUDA(cudaEventRecord(c->ev_join[half], c->st2));
  // h = M p is kept by the recurrence h_new = M r + gammag h_old (p = r + gammag p
  // and linearity), so p is never formed: the M launch reads the newest residual,
  // the previous h and the links and writes h (|h|^2 from registers); the
  // M^dagger launch reads h, the links and r_old and writes r_new.  The two h
  // fields alternate (hv on even iterations, p's field on odd ones; kBatch is even).
  // M sweeps up and M^dagger down, so each starts on the sites the other wrote last.
  const double b_md = 3.0 * n * sizeof(V) + 3.0 * c->g.v3 * lb;
  MsHist* rec = hist + half;
  const int rev_md = c->rev_sweep ? 1 : 0;
  (void)gb;
  // FP64 on a small lattice: the batch as one persistent kernel (msp.cu), same recurrences
  if constexpr (sizeof(V) == sizeof(double2) && sizeof(VO) == sizeof(double2)) {
    if (!prof && ms_chain_batch(c, ms, rec, nullptr, nullptr, nullptr, am, imass, half, main, true) == THR_OK) {
      THR_TRY(ms_chain_batch(c, ms, rec, reinterpret_cast<double2*>(ring), reinterpret_cast<double2*>(hv),
                             reinterpret_cast<double2*>(p), am, imass, half, main, false));
      if (fork) THR_CUDA(cudaStreamWaitEvent(main, c->ev_join[half], 0));
      return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
    }
  }
  for (int j = 0; j < kBatch; j++) {
    const int so = half * kBatch + j, sn = so + 1 == 2 * kBatch ? 0 : so + 1;
    V* rold = ring + (size_t)so * n;
    V* rnew = ring + (size_t)sn * n;
    V* hcur = (j & 1) ? p : hv;
    const V* hprev = (j & 1) ? hv : p;
    // alpha = Re<p, M^dagger M p> (:104) evaluated as |h|^2 = |M p|^2 in the M epilogue
    // each kernel of the chain is a dependent launch of the one before (not across a sampled
    // launch's events, nor for the batch's first, which follows the flush fork)
    int pe = prof ? c->prof_begin(fp64 ? thr_ctx::P_DSLASH : thr_ctx::P_DSLASH_LOW, b_md, k0 + j) : -1;
    THR_TRY(launch_dslash_accum<V>(c->g, c->p.kernel, false, hcur, rold, u, am, imass, c->p.am3, main, &ms->done,
                                   hprev, &ms->gammag, c->partials, 0, pdl && j > 0));
    c->prof_end(pe);
    pe = prof ? c->prof_begin(thr_ctx::P_ALPHA, 0.0, k0 + j) : -1;
    launch_k(k_alpha, dim3(1), dim3(1024), 0, main, pdl, ms, rec, c->partials, (int)gs);
    c->prof_end(pe);
    // s = M^dagger h is never stored: the epilogue forms r = r + omega*s (:137) and |r|^2 (:138)
    pe = prof ? c->prof_begin(fp64 ? thr_ctx::P_DSLASH_DAG : thr_ctx::P_DSLASH_DAG_LOW, b_md, k0 + j) : -1;
    THR_TRY(launch_dslash_axpy<V>(c->g, c->p.kernel, true, rnew, hcur, u, am, imass, c->p.am3, main, &ms->done,
                                  rold, &ms->omega, c->partials, rev_md, pdl));
    c->prof_end(pe);
    pe = prof ? c->prof_begin(thr_ctx::P_LAMBDA, 0.0, k0 + j) : -1;
    launch_k(k_lambda, dim3(1), dim3(1024), 0, main, pdl, ms, rec, c->partials, (int)gs);
    c->prof_end(pe);
  }
  (void)s;
  if (fork) THR_CUDA(cudaStreamWaitEvent(main, c->ev_join[half], 0));
  return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
}

// The whole batch loop as one CUDA graph: a WHILE conditional node whose body is
// two batches (ring halves 0 and 1, each with the other half's flush alongside)
// followed by k_loop_ctl, then the flush of the last half-1 batch.  The body reads
// every per-solve value from device memory (MsState), so one instantiated graph
// serves every solve with the same buffers and operator; it is rebuilt when they
// change.
struct MsGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  const void *out = nullptr, *sf = nullptr, *ring = nullptr, *p = nullptr, *hv = nullptr, *s = nullptr;
  const void *u = nullptr, *partials = nullptr, *ms = nullptr, *hist = nullptr, *cf = nullptr;
  float am = 0.f, am3 = 0.f;
  int imass = 0, kernel = -1;
  size_t n = 0;
  void release() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
};

// graph cache slot of a (base storage, shift field) pair
template <class V, class VO> constexpr int graph_slot() {
  return sizeof(VO) == sizeof(float2) ? 1 : sizeof(V) == sizeof(double2) ? 0 : sizeof(V) == sizeof(float2) ? 2 : 3;
}

template <class V, class VO = V>
int ms_graph_build(thr_ctx* c, MsState* ms, MsHist* hist, MsCoef* cf, VO* out, VO* sf, V* ring, V* p, V* hv, V* s,
                   float am, int imass, cudaGraphExec_t* exec_out);

// the cached graph, built if needed; a build with dependent launches that the driver
// rejects is retried without them (they are then off for the context)
template <class V, class VO = V>
int ms_graph(thr_ctx* c, MsState* ms, MsHist* hist, MsCoef* cf, VO* out, VO* sf, V* ring, V* p, V* hv, V* s, float am,
             int imass, cudaGraphExec_t* exec_out) {
  int rc = ms_graph_build<V, VO>(c, ms, hist, cf, out, sf, ring, p, hv, s, am, imass, exec_out);
  // a graph that cannot be built with the persistent batch kernel's cooperative
  // launches, or then with dependent launches, is built without them
  if (rc != THR_OK && c->chain_mode != 0) {
    c->chain_mode = 0;
    rc = ms_graph_build<V, VO>(c, ms, hist, cf, out, sf, ring, p, hv, s, am, imass, exec_out);
  }
  if (rc != THR_OK && c->use_pdl) {
    c->use_pdl = false;
    rc = ms_graph_build<V, VO>(c, ms, hist, cf, out, sf, ring, p, hv, s, am, imass, exec_out);
  }
  return rc;
}

template <class V, class VO>
int ms_graph_build(thr_ctx* c, MsState* ms, MsHist* hist, MsCoef* cf, VO* out, VO* sf, V* ring, V* p, V* hv, V* s,
                   float am, int imass, cudaGraphExec_t* exec_out) {
  const int slot = graph_slot<V, VO>();
  if (!c->ms_graphs[slot]) c->ms_graphs[slot] = new MsGraph();
  MsGraph& G = *static_cast<MsGraph*>(c->ms_graphs[slot]);
  const void* u = sizeof(V) == sizeof(double2) ? (const void*)c->u64 : (const void*)c->u32;
  if (G.exec && G.out == out && G.sf == sf && G.ring == ring && G.p == p && G.hv == hv && G.s == s && G.u == u &&
      G.partials == c->partials && G.ms == ms && G.hist == hist && G.cf == cf && G.am == am && G.am3 == c->p.am3 && G.imass == imass &&
      G.kernel == c->p.kernel && G.n == c->n4()) {
    *exec_out = G.exec;
    return THR_OK;
  }
  G.release();
  // run the two stencils of an iteration once outside the capture, so that the
  // autotuner settles their configuration before it is baked into the graph
  // (hv, p, s and the partials are scratch at this point; the solve clears hv and p after)
  {
    const typename Sto<V>::C* uu = (const typename Sto<V>::C*)u;
    THR_TRY(launch_dslash_accum<V>(c->g, c->p.kernel, false, hv, ring, uu, am, imass, c->p.am3, c->st, &ms->done, p,
                                   &ms->gammag, c->partials, 0));
    THR_TRY(launch_dslash_axpy<V>(c->g, c->p.kernel, true, s, hv, uu, am, imass, c->p.am3, c->st, &ms->done, ring,
                                  &ms->omega, c->partials, c->rev_sweep ? 1 : 0));
  }
  THR_CUDA(cudaGraphCreate(&G.graph, 0));
  cudaGraphConditionalHandle handle;
  THR_CUDA(cudaGraphConditionalHandleCreate(&handle, G.graph, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  THR_CUDA(cudaGraphAddNode(&node, G.graph, nullptr, 0, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  THR_CUDA(cudaStreamBeginCaptureToGraph(c->st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_batch<V, VO>(c, ms, hist, cf, out, sf, ring, p, hv, s, am, imass, 0, 0, false, nullptr, c->st);
  if (rc == THR_OK)
    rc = enqueue_batch<V, VO>(c, ms, hist, cf, out, sf, ring, p, hv, s, am, imass, 1, 0, false, nullptr, c->st);
  if (rc == THR_OK) k_loop_ctl<<<1, 1, 0, c->st>>>(ms, handle);
  cudaGraph_t captured = nullptr;
  cudaError_t ce = cudaStreamEndCapture(c->st, &captured);
  if (rc == THR_OK && ce == cudaSuccess) {
    // after the loop: the flush of the last batch (ring half 1)
    ce = cudaStreamBeginCaptureToGraph(c->st, G.graph, &node, nullptr, 1, cudaStreamCaptureModeThreadLocal);
    if (ce == cudaSuccess) {
      enqueue_flush<V, VO>(c, c->st, ms, hist + 1, cf + 1, out, sf, ring, 1, false, 0, nullptr);
      ce = cudaStreamEndCapture(c->st, &captured);
    }
  }
  if (rc != THR_OK || ce != cudaSuccess) {
    G.release();
    cudaGetLastError();
    return rc != THR_OK ? rc : THR_ERR_CUDA;
  }
  // node priorities: the flush nodes captured from the side stream yield to the main chain
  if (cudaGraphInstantiate(&G.exec, G.graph, cudaGraphInstantiateFlagUseNodePriority) != cudaSuccess) {
    G.release();
    cudaGetLastError();
    return THR_ERR_CUDA;
  }
  G.out = out; G.sf = sf; G.ring = ring; G.p = p; G.hv = hv; G.s = s; G.u = u;
  G.partials = c->partials; G.ms = ms; G.hist = hist; G.cf = cf; G.am = am; G.am3 = c->p.am3; G.imass = imass;
  G.kernel = c->p.kernel; G.n = c->n4();
  *exec_out = G.exec;
  return THR_OK;
}
}  // namespace

void ms_graphs_release(thr_ctx* c) {
  for (void*& g : c->ms_graphs) {
    if (g) {
      static_cast<MsGraph*>(g)->release();
      delete static_cast<MsGraph*>(g);
      g = nullptr;
    }
  }
}

namespace {
// double2 -> the low-precision storage of the mixed solver's second phase (round to nearest)
__device__ __forceinline__ void narrow(float2* d, double2 v) { *d = make_float2((float)v.x, (float)v.y); }
__device__ __forceinline__ void narrow(__nv_bfloat162* d, double2 v) {
  *d = __float22bfloat162_rn(make_float2((float)v.x, (float)v.y));
}
template <class VL>
__global__ void k_narrow(VL* d, const double2* s, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    narrow(d + i, s[i]);
}
__global__ void k_end_phase(MsState* ms) { ms->switch_delta = 0.0; }

// Runs batches (base storage V, shift fields VO) from the device state until the solve
// is done or -- when the state's switch_delta is set -- the base residual falls below
// it (tested after each pair of batches, in the graph and on the host alike); ends
// with the last batch's flush.  `prime` runs after the graph is built and before the
// first batch (it sets up the h fields).  The state after the run is left in *h.
template <class V, class VO, class Prime>
int run_batches(thr_ctx* c, MsState* ms, MsState* h, MsHist* hist, MsCoef* cf, VO* out, VO* sf, V* ring, V* p, V* hv,
                V* s, float am, int imass, Prime&& prime) {
  const size_t n = c->n4();
  if (c->md_capture) {
    // inside a captured MD step: the batch loop becomes a WHILE node of the graph
    // being captured on c->st, its body captured on c->st3; nothing is read back
    THR_TRY(prime());
    cudaStreamCaptureStatus cst;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    THR_CUDA(cudaStreamGetCaptureInfo(c->st, &cst, nullptr, &g, &deps, &nd));
    if (cst != cudaStreamCaptureStatusActive) return THR_ERR_CUDA;
    cudaGraphConditionalHandle handle;
    THR_CUDA(cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    THR_CUDA(cudaGraphAddNode(&node, g, deps, nd, &cp));
    THR_CUDA(cudaStreamUpdateCaptureDependencies(c->st, &node, 1, cudaStreamSetCaptureDependencies));
    THR_CUDA(cudaStreamBeginCaptureToGraph(c->st3, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_batch<V, VO>(c, ms, hist, cf, out, sf, ring, p, hv, s, am, imass, 0, 0, false, nullptr, c->st3);
    if (rc == THR_OK)
      rc = enqueue_batch<V, VO>(c, ms, hist, cf, out, sf, ring, p, hv, s, am, imass, 1, 0, false, nullptr, c->st3);
    if (rc == THR_OK) k_loop_ctl<<<1, 1, 0, c->st3>>>(ms, handle);
    cudaGraph_t body = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(c->st3, &body);
    if (rc != THR_OK) return rc;
    if (ce != cudaSuccess) return THR_ERR_CUDA;
    // the last batch's flush (ring half 1), after the loop, on the captured stream
    enqueue_flush<V, VO>(c, c->st, ms, hist + 1, cf + 1, out, sf, ring, 1, false, 0, nullptr);
    return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
  }
  if (c->use_graphs && !c->prof_on) {
    // one graph launch runs every batch until convergence (or the switch); one synchronisation
    cudaGraphExec_t exec = nullptr;
    THR_TRY(ms_graph<V, VO>(c, ms, hist, cf, out, sf, ring, p, hv, s, am, imass, &exec));
    THR_TRY(prime());
    THR_CUDA(cudaGraphLaunch(exec, c->st));
    THR_CUDA(cudaMemcpyAsync(h, ms, sizeof(MsState), cudaMemcpyDeviceToHost, c->st));
    THR_CUDA(cudaStreamSynchronize(c->st));
    return THR_OK;
  }
  // stream-launched batches, one synchronisation per batch (and kernel timing)
  THR_TRY(prime());
  const size_t prof_first = c->prof_kind.size();
  THR_CUDA(cudaMemcpyAsync(h, ms, sizeof(MsState), cudaMemcpyDeviceToHost, c->st));
  THR_CUDA(cudaStreamSynchronize(c->st));
  const long long it0 = h->it;
  double flushed = h->flush_fields;
  long long flushes = 0;
  // flush traffic: each recorded step's residual read once, each shift field of the
  // batch's window read and written once (out and sf), counted at the shift fields' width
  auto account = [&](int pf) {
    c->prof_set_bytes(pf, (h->flush_fields - flushed) * n * sizeof(VO));
    if (h->flush_fields > flushed) flushes++;
    flushed = h->flush_fields;
  };
  int half = 0;
  for (long long k = it0;; k += kBatch, half ^= 1) {
    int pf = -1;
    THR_TRY(
        enqueue_batch<V, VO>(c, ms, hist, cf, out, sf, ring, p, hv, s, am, imass, half, k, c->prof_on, &pf, c->st));
    THR_CUDA(cudaMemcpyAsync(h, ms, sizeof(MsState), cudaMemcpyDeviceToHost, c->st));
    THR_CUDA(cudaStreamSynchronize(c->st));
    account(pf);
    const bool sw = half == 1 && h->switch_delta > 0.0 && h->delta < h->switch_delta;
    if (h->done || sw) {
      // the last batch's own flush
      enqueue_flush<V, VO>(c, c->st, ms, hist + half, cf + half, out, sf, ring, half, c->prof_on, k, &pf);
      THR_CUDA(cudaMemcpyAsync(h, ms, sizeof(MsState), cudaMemcpyDeviceToHost, c->st));
      THR_CUDA(cudaStreamSynchronize(c->st));
      account(pf);
      break;
    }
    if (h->batches >= h->max_batches) return THR_ERR_CUDA;  // the device state stopped advancing
  }
  if (c->prof_on) {
    const bool fp64 = sizeof(V) == sizeof(double2);
    c->prof_trim(prof_first, h->it);  // launches after convergence skipped their work
    c->prof_work[fp64 ? thr_ctx::P_DSLASH : thr_ctx::P_DSLASH_LOW] += h->it - it0;
    c->prof_work[fp64 ? thr_ctx::P_DSLASH_DAG : thr_ctx::P_DSLASH_DAG_LOW] += h->it - it0;
    c->prof_work[thr_ctx::P_SHIFTUPD] += flushes;
    c->prof_work[thr_ctx::P_ALPHA] += h->it - it0;
    c->prof_work[thr_ctx::P_LAMBDA] += h->it - it0;
  }
  return THR_OK;
}

// state, histories and coefficient tables of a batched solve; r = input in ring slot 0,
// delta = |input|^2, out = 0, sf = input
template <class V>
int batched_setup(thr_ctx* c, const V* in, V* out, V* sf, V* ring, int ndiagq, const double* aden, const double* anum,
                  float res, int maxcg, double switch_rel, MsState** ms_out, MsState** h_out, MsHist** hist_out,
                  MsCoef** cf_out) {
  const size_t n = c->n4();
  MsState* ms = reinterpret_cast<MsState*>(c->dscal);
  // the initial state is copied from host memory when the copy runs: inside a captured MD
  // step every solve gets its own pinned template, which stays valid for the graph's life
  MsState* h = reinterpret_cast<MsState*>(c->hscal);
  if (c->md_capture) {
    if (c->ms_tmpl_next >= kMsTemplates) return THR_ERR_BADSHAPE;
    h = reinterpret_cast<MsState*>(c->ms_tmpl) + c->ms_tmpl_next++;
  }
  void* hv_;
  THR_TRY(c->buffer(thr_ctx::B_HIST, 2 * sizeof(MsHist), &hv_));
  void* cf_;
  THR_TRY(c->buffer(thr_ctx::B_COEF, 2 * sizeof(MsCoef), &cf_));
  MsHist* hist = (MsHist*)hv_;  // one history per ring half
  THR_TRY(ms_prepare_state(c, h, ndiagq, aden, anum, res, maxcg));
  h->kbase = 0;
  h->batches = 0;
  // flushes (one per batch, plus the final one; the graph runs batches in pairs)
  h->max_batches = (maxcg > 0 ? maxcg : 0) / kBatch + 5;
  h->switch_rel2 = switch_rel * switch_rel;
  THR_CUDA(cudaMemcpyAsync(ms, h, sizeof(MsState), cudaMemcpyHostToDevice, c->st));
  THR_CUDA(cudaMemcpyAsync(ring, in, n * sizeof(V), cudaMemcpyDeviceToDevice, c->st));  // r = input (slot 0)
  const unsigned gb = vec_grid(n);
  k_norm2<V><<<gb, kThreads, 0, c->st>>>(ring, n, c->partials);
  k_init<<<1, kThreads, 0, c->st>>>(ms, hist, c->partials, gb);
  THR_CUDA(cudaMemsetAsync(out, 0, (size_t)ndiagq * n * sizeof(V), c->st));
  k_fill<V><<<gb, kThreads, 0, c->st>>>(sf, in, n, n, ndiagq);
  *ms_out = ms;
  *h_out = h;
  *hist_out = hist;
  *cf_out = (MsCoef*)cf_;
  return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
}
}  // namespace

template <class V>
int multishift_batched_dev(thr_ctx* c, const V* in, V* out, V* sf, V* ring, V* p, V* hv, V* s, int ndiagq,
                           const double* aden, const double* anum, float res, float am, int imass, int maxcg,
                           int* cg_return, int* cg_returns) {
  const size_t n = c->n4();
  MsState *ms, *h;
  MsHist* hist;
  MsCoef* cf;
  THR_TRY(batched_setup<V>(c, in, out, sf, ring, ndiagq, aden, anum, res, maxcg, 0.0, &ms, &h, &hist, &cf));
  // h = M p starts as M r (p = r, gammag = 0): the previous h of the first iteration is zero
  auto prime = [&]() -> int {
    THR_CUDA(cudaMemsetAsync(hv, 0, n * sizeof(V), c->st));
    THR_CUDA(cudaMemsetAsync(p, 0, n * sizeof(V), c->st));
    return THR_OK;
  };
  THR_TRY(run_batches<V, V>(c, ms, h, hist, cf, out, sf, ring, p, hv, s, am, imass, prime));
  if (c->md_capture) return THR_OK;  // the results stay on the device
  if (cg_return) *cg_return = h->it;
  if (cg_returns)
    for (int q = 0; q < ndiagq; q++) cg_returns[q] = h->cg_returns[q];
  return h->status ? h->status : THR_OK;
}

// Mixed precision.  FP32 (or BF16) rounding of the base iteration enters every shifted
// solution with the size of the base residual at the time it is made, and the shifted
// systems have no residual of their own that could correct it later; so the solve runs
// in FP64 while |r| is large and moves the base iteration to low precision only once
// |r| < switch_rel |input|, where that rounding stays below FP64's own.  The shift
// fields out and sf stay FP64 throughout: the flush widens the low-precision residuals.
// The precision changes between two pairs of batches: the FP64 ring's last residual
// (slot 0) and h (in p) are rounded into the low-precision ring's slot 0 and h field,
// and the recurrences continue.
template <class VL>
int multishift_mixed_dev(thr_ctx* c, const double2* in, double2* out, double2* sf, double2* ring64, double2* p,
                         double2* hv, double2* s, VL* low, int ndiagq, const double* aden, const double* anum,
                         float res, float am, int imass, int maxcg, double switch_rel, int* cg_return,
                         int* cg_returns, int* switched_at) {
  const size_t n = c->n4();
  MsState *ms, *h;
  MsHist* hist;
  MsCoef* cf;
  THR_TRY(batched_setup<double2>(c, in, out, sf, ring64, ndiagq, aden, anum, res, maxcg, switch_rel, &ms, &h, &hist,
                                 &cf));
  auto prime64 = [&]() -> int {
    THR_CUDA(cudaMemsetAsync(hv, 0, n * sizeof(double2), c->st));
    THR_CUDA(cudaMemsetAsync(p, 0, n * sizeof(double2), c->st));
    return THR_OK;
  };
  if (c->md_capture) return THR_ERR_UNSUPPORTED;  // the precision switch is decided on the host
  THR_TRY(run_batches<double2, double2>(c, ms, h, hist, cf, out, sf, ring64, p, hv, s, am, imass, prime64));
  if (switched_at) *switched_at = 0;
  if (!h->done && !h->status) {
    // the low-precision ring occupies the upper half of the FP64 ring's memory
    // (2 kBatch fields of n VL are at most kBatch FP64 fields), clear of slot 0
    VL* ring = reinterpret_cast<VL*>(ring64 + (size_t)kBatch * n);
    VL *pl = low, *hl = low + n, *sl = low + 2 * n;
    if (switched_at) *switched_at = h->it;
    auto prime = [&]() -> int {
      const unsigned gb = vec_grid(n);
      k_narrow<VL><<<gb, kThreads, 0, c->st>>>(ring, ring64, n);  // latest residual, slot 0
      k_narrow<VL><<<gb, kThreads, 0, c->st>>>(pl, p, n);         // latest h (odd iterations write p)
      k_end_phase<<<1, 1, 0, c->st>>>(ms);
      return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
    };
    THR_TRY(run_batches<VL, double2>(c, ms, h, hist, cf, out, sf, ring, pl, hl, sl, am, imass, prime));
  }
  if (cg_return) *cg_return = h->it;
  if (cg_returns)
    for (int q = 0; q < ndiagq; q++) cg_returns[q] = h->cg_returns[q];
  return h->status ? h->status : THR_OK;
}

template int multishift_mixed_dev<float2>(thr_ctx*, const double2*, double2*, double2*, double2*, double2*, double2*,
                                          double2*, float2*, int, const double*, const double*, float, float, int,
                                          int, double, int*, int*, int*);
template int multishift_mixed_dev<__nv_bfloat162>(thr_ctx*, const double2*, double2*, double2*, double2*, double2*,
                                                  double2*, double2*, __nv_bfloat162*, int, const double*,
                                                  const double*, float, float, int, int, double, int*, int*, int*);

template int multishift_batched_dev<double2>(thr_ctx*, const double2*, double2*, double2*, double2*, double2*,
                                             double2*, double2*, int, const double*, const double*, float, float, int,
                                             int, int*, int*);
template int multishift_batched_dev<float2>(thr_ctx*, const float2*, float2*, float2*, float2*, float2*, float2*,
                                            float2*, int, const double*, const double*, float, float, int, int, int*,
                                            int*);

}  // namespace thr
