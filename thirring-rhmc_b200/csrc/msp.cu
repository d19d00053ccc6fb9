// msp.cu -- one batch of the batched multishift as one persistent kernel (small lattices).
//
// On a small lattice every kernel of the batched solver's iteration chain (msb.cu:
// M with the h recurrence, the alpha step, M^dagger with the residual update, the
// lambda step) runs for 2-3 us, and the chain is bound by the launches between them.
// Here one cooperative launch runs a whole batch (kBatch iterations of one ring half):
// its blocks own the stencil's site blocks (one partial each, as the stencil kernel's
// blocks), and two grid barriers per iteration separate the stencils from the sums
// that follow them.  Every block keeps its own copy of the solver state in shared
// memory and runs the scalar steps itself (ms_alpha_block / ms_lambda_block on the
// same partials, summed in the order block_sum_partials uses with 1024 threads), so
// no block waits for another's scalars and all copies stay identical; block 0 alone
// records the batch's coefficients and writes the state back.  The stencils are
// dslash_block with loads through L2 (the fields are rewritten during the launch), so
// per site the instructions are the stencil kernel's.  The flush of the batch, the
// loop control and the mixed-precision switch stay as in msb.cu.
//
// Barriers count arrivals in bar[0] (the k-th barrier of a launch completes at
// k * gridDim.x), bar[1] counts the blocks that have finished, and the last one to
// finish clears the words for the next launch.  Every wait is bounded: after
// kBarrierNs of global time a block raises bar[2]; a block that sees bar[2] raised
// leaves the batch, and block 0 then reports THR_ERR_TIMEOUT in the solver state
// (which ends the solve) instead of writing the state back.
#include <algorithm>
#include <atomic>
#include <cstdlib>

#include "ctx.h"
#include "dslash_site.cuh"
#include "ms.h"
#include "thr_kernels.h"

namespace thr {

namespace {
constexpr unsigned long long kBarrierNs = 200000000ull;  // 0.2 s of global time per wait

__device__ __forceinline__ unsigned long long chain_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// true once every block of the grid has arrived (bar[0] >= target); false if the wait
// ran out or another block gave up first.  Thread 0 arrives with a release pattern
// (fence.acq_rel.gpu, then a relaxed add) after the block's __syncthreads, and polls
// with acquire loads; the closing __syncthreads hands the acquired view to the block.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned target, int tid) {
  __shared__ int ok;
  __syncthreads();
  if (tid == 0) {
    asm volatile("fence.acq_rel.gpu;\n\tred.relaxed.gpu.global.add.u32 [%0], 1;" ::"l"(bar) : "memory");
    int r = 1;
    const unsigned long long t0 = chain_ns();
    unsigned polls = 0;
    while (ld_acquire(bar) < target) {
      if (ld_acquire(bar + 2)) {
        r = 0;
        break;
      }
      if ((++polls & 255u) == 0 && chain_ns() - t0 > kBarrierNs) {
        atomicExch(bar + 2, 1u);
        r = 0;
        break;
      }
    }
    ok = r;
  }
  __syncthreads();
  return ok != 0;
}

// The partials of a stencil pass, written by every block, are copied into shared memory
// with cp.async (16 bytes each, through L2) right after the barrier, while the block
// computes its next stencil pass; the sum waits for them only when its result is due.
constexpr int kChainMaxParts = 2048;  // partials one block stages (stencil site blocks)
__device__ __forceinline__ void stage_partials(double* sp, const double* p, int n, int tid, int nthr) {
  const int n2 = (n + 1) & ~1;  // the arrays are padded to an even length
  for (int i = 2 * tid; i < n2; i += 2 * nthr) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(sp + i);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(p + i) : "memory");
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}

// block_sum_partials(p, n) as a block of 1024 threads computes it, by the whole warps of
// this block, from the staged copy sp: virtual thread i sums sp[i], sp[i + 1024], ... in
// order, each virtual warp's 32 values go through the same shuffle tree, then the 32 warp
// sums.  Waits for the staging copies first.
__device__ __forceinline__ double sum_staged(const double* sp, int n, int tid, int nthr, double* sh) {
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();
  const int lane = tid & 31, warp = tid >> 5, nwarps = nthr >> 5;
  if (warp < nwarps) {
    for (int w = warp; w < 32; w += nwarps) {
      double v = 0.0;
      for (int i = w * 32 + lane; i < n; i += 1024) v += sp[i];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) sh[w] = v;
    }
  }
  __syncthreads();
  if (tid < 32) {
    double v = sh[tid];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (tid == 0) sh[32] = v;
  }
  __syncthreads();
  const double r = sh[32];
  __syncthreads();
  return r;
}

static_assert(sizeof(MsState) % sizeof(double) == 0, "MsState is copied as doubles");

struct ChainArgs {
  MsState* ms;
  MsHist* rec;
  double2* ring;
  double2* hv;
  double2* p;
  const double2* u;
  Geom g;
  float am, am3;
  int imass;
  double* pa;  // partials of |h|^2 (alpha)
  double* pl;  // partials of |r|^2 (lambda); both arrays 16-byte aligned, padded to even length
  int np;      // stencil site blocks
  int half;    // ring half of the batch
  unsigned* bar;
  unsigned extra;  // added to every barrier's target (the timeout test); 0 in use
};

template <int KER, int NT, bool SHFL>
__global__ void __launch_bounds__(NT, 512 / NT) k_ms_chain(ChainArgs a) {
  using C = double2;
  __shared__ MsState st;
  __shared__ __align__(16) double sp[kChainMaxParts];
  __shared__ double sh[33];
  __shared__ int s_lo, s_hi;
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int nthr = blockDim.x * blockDim.y;
  {
    const double* src = reinterpret_cast<const double*>(a.ms);
    double* dst = reinterpret_cast<double*>(&st);
    for (int i = tid; i < (int)(sizeof(MsState) / sizeof(double)); i += nthr) dst[i] = __ldcg(src + i);
  }
  const int nstep0 = __ldcg(&a.rec->nsteps);
  __syncthreads();
  const Geom g = a.g;
  const size_t n = 4 * (size_t)g.v5;
  const bool lead = blockIdx.x == 0;
  MsHist* rec = lead ? a.rec : nullptr;
  unsigned target = a.extra;
  bool ok = true;
  int nstep = nstep0;
  bool lam_due = false;  // the lambda step of the iteration before is still to be taken
  for (int j = 0;; j++) {
    if (j == kBatch || (!lam_due && st.done)) {
      if (lam_due) {
        ms_lambda_block(&st, rec, nstep, sum_staged(sp, a.np, tid, nthr, sh), tid, &s_lo, &s_hi);
        __syncthreads();
        nstep++;
      }
      break;
    }
    const int so = a.half * kBatch + j, sn = so + 1 == 2 * kBatch ? 0 : so + 1;
    const double2* rold = a.ring + (size_t)so * n;
    double2* rnew = a.ring + (size_t)sn * n;
    double2* hcur = (j & 1) ? a.p : a.hv;
    const double2* hprev = (j & 1) ? a.hv : a.p;
    // h = M r + gammag h_prev and the partials of |h|^2 (alpha = |M p|^2, :104); the
    // previous iteration's lambda step runs between the first site block's stencil and
    // its epilogue, which is the first use of gammag.  If that step ends the solve, the
    // stencil's result is dropped, as the kernel chain does not run it.
    bool first = true, stop = false;
    for (int t = blockIdx.x; t < a.np; t += gridDim.x) {
      C acc[4];
      block_sites<double2, KER, false, SHFL, true>(rold, a.u, g, a.am, a.imass, a.am3, t, acc);
      if (first) {
        first = false;
        if (lam_due) {
          ms_lambda_block(&st, rec, nstep, sum_staged(sp, a.np, tid, nthr, sh), tid, &s_lo, &s_hi);
          __syncthreads();
          nstep++;
          lam_due = false;
        }
        if (st.done) {
          stop = true;
          break;
        }
      }
      const int site = t * blockDim.y + threadIdx.y;
      double racc = 0.0;
      if (site < g.v3) {
#pragma unroll
        for (int d = 0; d < 4; d++)
          epi_element<double2, 3, true>(hcur, hprev, st.gammag, sidx32(g, threadIdx.x, site, d), acc[d], racc);
      }
      block_partial_sum<NT>(racc, a.pa, t);
      __syncthreads();
    }
    if (stop) break;
    target += gridDim.x;
    if (!(ok = grid_barrier(a.bar, target, tid))) break;
    stage_partials(sp, a.pa, a.np, tid, nthr);
    // r_new = r_old + omega M^dagger h (:137) and the partials of |r_new|^2 (:138); the
    // alpha step runs between the first site block's stencil and its epilogue
    first = true;
    for (int t = blockIdx.x; t < a.np; t += gridDim.x) {
      C acc[4];
      block_sites<double2, KER, true, SHFL, true>(hcur, a.u, g, a.am, a.imass, a.am3, t, acc);
      if (first) {
        first = false;
        ms_alpha_block(&st, rec, nstep, sum_staged(sp, a.np, tid, nthr, sh), tid);
        __syncthreads();
      }
      const int site = t * blockDim.y + threadIdx.y;
      double racc = 0.0;
      if (site < g.v3) {
#pragma unroll
        for (int d = 0; d < 4; d++)
          epi_element<double2, 1, true>(rnew, rold, st.omega, sidx32(g, threadIdx.x, site, d), acc[d], racc);
      }
      block_partial_sum<NT>(racc, a.pl, t);
      __syncthreads();
    }
    target += gridDim.x;
    if (!(ok = grid_barrier(a.bar, target, tid))) break;
    stage_partials(sp, a.pl, a.np, tid, nthr);
    lam_due = true;
  }
  asm volatile("cp.async.wait_all;" ::: "memory");  // no copy outlives the block
  if (lead) {
    __shared__ int gave_up;
    if (tid == 0) gave_up = (!ok || ld_acquire(a.bar + 2)) ? 1 : 0;
    __syncthreads();
    MsState* m = a.ms;
    if (gave_up) {
      if (tid == 0) {
        m->status = THR_ERR_TIMEOUT;
        m->done = 1;
      }
    } else {
      // the fields an iteration changes (not batches or flush_fields: the side stream's
      // flush of the other ring half updates those meanwhile)
      if (tid == 0) {
        m->omega = st.omega;
        m->gammag = st.gammag;
        m->delta = st.delta;
        m->alpha = st.alpha;
        m->lambda = st.lambda;
        m->omega_save = st.omega_save;
        m->it = st.it;
        m->lo = st.lo;
        m->hi = st.hi;
        m->done = st.done;
        m->status = st.status;
        m->active_sum = st.active_sum;
      }
      for (int k = tid; k < kMaxShift; k += nthr) {
        m->zeta_i[k] = st.zeta_i[k];
        m->zeta_ii[k] = st.zeta_ii[k];
        m->zeta_iii[k] = st.zeta_iii[k];
        m->omegas[k] = st.omegas[k];
        m->gammas[k] = st.gammas[k];
        m->flags[k] = st.flags[k];
        m->cg_returns[k] = st.cg_returns[k];
      }
    }
  }
  // the last block to finish clears the barrier words for the next launch
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    if (atomicAdd(a.bar + 1, 1u) == gridDim.x - 1) {
      a.bar[0] = 0u;
      a.bar[2] = 0u;
      a.bar[1] = 0u;
      __threadfence();
    }
  }
}

// co-resident blocks of a k_ms_chain instantiation on this device (cached per device)
template <int KER, int NT, bool SHFL>
int chain_capacity() {
  constexpr int kDevs = 64;
  static std::atomic<int> cache[kDevs];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 0;
  if (dev < kDevs) {
    const int v = cache[dev].load(std::memory_order_relaxed);
    if (v > 0) return v;
  }
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_ms_chain<KER, NT, SHFL>, NT, 0) != cudaSuccess) return 0;
  const int cap = occ * device_sms();
  if (dev < kDevs && cap > 0) cache[dev].store(cap, std::memory_order_relaxed);
  return cap;
}

template <int KER, int NT, bool SHFL>
int chain_launch(thr_ctx* c, const ChainArgs& a, dim3 blk, cudaStream_t st, bool dry) {
  const int cap = chain_capacity<KER, NT, SHFL>();
  if (cap <= 0) return THR_ERR_UNSUPPORTED;
  // auto (mode 1): only where every site block has its own resident block; forced (2): any size
  if (c->chain_mode == 1 && a.np > cap) return THR_ERR_UNSUPPORTED;
  if (dry) return THR_OK;
  const unsigned grid = (unsigned)std::min(a.np, cap);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = blk;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_ms_chain<KER, NT, SHFL>, a) == cudaSuccess ? THR_OK : THR_ERR_CUDA;
}

// THR_CHAIN_WAIT_TEST=1: every barrier expects one arrival more than the grid has, so
// each wait runs out (a test of the timeout path: nothing is left waiting on the GPU)
unsigned chain_extra() {
  static const unsigned extra = [] {
    const char* e = std::getenv("THR_CHAIN_WAIT_TEST");
    return (e && e[0] == '1' && e[1] == 0) ? 1u : 0u;
  }();
  return extra;
}
}  // namespace

int ms_chain_batch(thr_ctx* c, MsState* ms, MsHist* rec, double2* ring, double2* hv, double2* p, float am, int imass,
                   int half, cudaStream_t st, bool dry) {
  if (c->chain_mode == 0) return THR_ERR_UNSUPPORTED;
  const Geom& g = c->g;
  const int kernel = c->p.kernel;
  const dim3 blk = stencil_block(g, kernel);
  const int nthr = (int)(blk.x * blk.y);
  const int np = (int)stencil_grid(g, kernel);
  // the block shapes of the stencil kernels' common configurations (128-thread Shamir,
  // 256-thread Wilson blocks) with at least nt / 32 - 1 whole warps (the sums' layout,
  // sum_staged) and kMaxShift threads (the scalar steps)
  const int nt = kernel == 0 ? 128 : 256;
  if (g.ls > nt || nthr > nt || nthr / 32 < nt / 32 - 1 || nthr < kMaxShift) return THR_ERR_UNSUPPORTED;
  const size_t npad = ((size_t)np + 1) & ~(size_t)1;  // pl 16-byte aligned, both arrays even
  if (np > kChainMaxParts || 2 * npad > c->nparts) return THR_ERR_UNSUPPORTED;
  ChainArgs a;
  a.ms = ms;
  a.rec = rec;
  a.ring = ring;
  a.hv = hv;
  a.p = p;
  a.u = c->u64;
  a.g = g;
  a.am = am;
  a.am3 = c->p.am3;
  a.imass = imass;
  a.pa = c->partials;
  a.pl = c->partials + npad;
  a.np = np;
  a.half = half;
  a.bar = reinterpret_cast<unsigned*>(c->iscal + kIscalChainBar);
  a.extra = chain_extra();
  const bool shfl = kernel == 0 && g.ls <= 32 && (g.ls & (g.ls - 1)) == 0;
  if (kernel == 1) return chain_launch<1, 256, false>(c, a, blk, st, dry);
  if (shfl) return chain_launch<0, 128, true>(c, a, blk, st, dry);
  return chain_launch<0, 128, false>(c, a, blk, st, dry);
}

}  // namespace thr
