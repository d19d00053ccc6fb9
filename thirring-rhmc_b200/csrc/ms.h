// ms.h -- multishift solver state (multishift_module.F90:43-57), device-resident.
#pragma once
#include "ctx.h"

namespace thr {

constexpr int kMaxShift = 64;

struct MsState {
  double omega, gammag, delta, alpha, lambda, omega_save;
  int it, maxcg, lo, hi, done, status, ndiagq;
  float res;
  double active_sum;    // sum over iterations of the shifts updated (for traffic accounting)
  double flush_fields;  // fields moved by the batched shift updates (for traffic accounting)
  long long kbase;      // batched solver: first iteration of the current batch (ring slot base)
  int batches, max_batches;  // batched solver: batches run, and the bound on them
  // mixed precision (batched solver): the FP64 phase ends once delta = |r|^2 falls
  // below switch_delta = switch_rel2 * |input|^2 (0: never)
  double switch_rel2, switch_delta;
  double zeta_i[kMaxShift], zeta_ii[kMaxShift], zeta_iii[kMaxShift];
  double omegas[kMaxShift], gammas[kMaxShift], correction[kMaxShift], aden[kMaxShift];
  int flags[kMaxShift], cg_returns[kMaxShift];
};
static_assert(sizeof(MsState) <= 4096 * sizeof(double), "MsState must fit the scalar block");

int ms_prepare_state(thr_ctx* c, MsState* h, int ndiagq, const double* aden, const double* anum, float res, int maxcg);

// ---- the scalar recurrences of multishift_module.F90, one statement group each
// iteration start and omega (:104, :126-127); one thread
__device__ __forceinline__ void ms_alpha_scalar(MsState* ms, double alpha) {
  ms->it += 1;
  ms->alpha = alpha;
  ms->omega_save = ms->omega;
  ms->omega = -ms->delta / alpha;
}
// zeta_iii and omegas of shift k (:129-135)
__device__ __forceinline__ void ms_alpha_shift(MsState* ms, int k) {
  const double omega = ms->omega, omega_save = ms->omega_save;
  ms->zeta_iii[k] = (ms->zeta_i[k] * ms->zeta_ii[k] * omega_save) /
                    (omega * ms->gammag * (ms->zeta_i[k] - ms->zeta_ii[k]) +
                     ms->zeta_i[k] * omega_save * (1.0 - ms->aden[k] * omega));
  ms->omegas[k] = omega * ms->zeta_iii[k] / ms->zeta_ii[k];
}
// lambda and gammag (:138-143); one thread
__device__ __forceinline__ void ms_lambda_scalar(MsState* ms, double lambda) {
  ms->lambda = lambda;
  ms->active_sum += (double)(ms->hi - ms->lo + 1);
  ms->gammag = lambda / ms->delta;
}
// gammas of shift k (:148-150)
__device__ __forceinline__ void ms_lambda_shift(MsState* ms, int k) {
  ms->gammas[k] = ms->gammag * ms->zeta_iii[k] * ms->omegas[k] / (ms->zeta_ii[k] * ms->omega);
}
// cg_returns, convergence test, window, zeta shift, delta (:178-180, :230-275); one thread
__device__ __forceinline__ void ms_converge_step(MsState* ms) {
  for (int k = ms->lo; k <= ms->hi; k++) ms->cg_returns[k] = ms->it;
  int maxi = -1, mini = ms->ndiagq;
  for (int k = 0; k < ms->ndiagq; k++) {
    if (ms->flags[k]) {
      if (sqrt(ms->delta * ms->zeta_ii[k] * ms->zeta_ii[k]) * ms->correction[k] < (double)ms->res) {
        ms->flags[k] = 0;
      } else {
        maxi = k > maxi ? k : maxi;
        mini = k < mini ? k : mini;
      }
    }
  }
  ms->lo = mini;
  ms->hi = maxi;
  for (int k = mini; k <= maxi; k++) {
    ms->zeta_i[k] = ms->zeta_ii[k];
    ms->zeta_ii[k] = ms->zeta_iii[k];
  }
  ms->delta = ms->lambda;
  if (!(ms->lambda == ms->lambda)) ms->status = THR_ERR_NAN;
  if (maxi < mini || ms->it >= ms->maxcg || ms->status) ms->done = 1;
}

// Batched variant: per-iteration coefficients of the shift update, applied
// every kBatch iterations in one pass over the shift fields.
constexpr int kBatch = 32;
struct MsHist {
  int nsteps;
  int lo[kBatch], hi[kBatch];
  double om[kBatch][kMaxShift], ga[kBatch][kMaxShift], ze[kBatch][kMaxShift];
};

// The batched solver's two scalar steps of an iteration, by the threads of one block
// (tid = 0 .. at least kMaxShift - 1, every thread of the block calls them).  rec (if not
// null) records the step's window and coefficients as step nstep of the batch.
// alpha known (:104): it, omega (:126-127), then zeta_iii and omegas per shift (:129-135)
__device__ __forceinline__ void ms_alpha_block(MsState* ms, MsHist* rec, int nstep, double alpha, int tid) {
  if (tid == 0) {
    ms_alpha_scalar(ms, alpha);
    if (rec) {
      rec->lo[nstep] = ms->lo;
      rec->hi[nstep] = ms->hi;
    }
  }
  __syncthreads();
  const int k = ms->lo + tid;
  if (k <= ms->hi) {
    ms_alpha_shift(ms, k);
    if (rec) {
      rec->om[nstep][k] = ms->omegas[k];
      rec->ze[nstep][k] = ms->zeta_iii[k];
    }
  }
}
// lambda known (:138): gammag (:143) and gammas per shift (:148-150); then the step's end
// (:178-180, :230-275: cg_returns, convergence test, window, zeta shift, delta) with one
// thread per shift -- ms_converge_step's statements, the window's new bounds from a
// min / max over the block in the shared s_lo, s_hi
__device__ __forceinline__ void ms_lambda_block(MsState* ms, MsHist* rec, int nstep, double lambda, int tid,
                                                int* s_lo, int* s_hi) {
  if (tid == 0) ms_lambda_scalar(ms, lambda);
  __syncthreads();
  const int lo0 = ms->lo, hi0 = ms->hi;
  const int k = lo0 + tid;
  if (k <= hi0) {
    ms_lambda_shift(ms, k);
    if (rec) rec->ga[nstep][k] = ms->gammas[k];
  }
  const int nq = ms->ndiagq, it = ms->it;
  const double delta = ms->delta, res = (double)ms->res;  // delta of this step (replaced below)
  if (tid == 0) {
    *s_lo = nq;
    *s_hi = -1;
  }
  __syncthreads();
  const int q = tid;
  if (q < nq) {
    if (q >= lo0 && q <= hi0) ms->cg_returns[q] = it;
    if (ms->flags[q]) {
      if (sqrt(delta * ms->zeta_ii[q] * ms->zeta_ii[q]) * ms->correction[q] < res) {
        ms->flags[q] = 0;
      } else {
        atomicMin(s_lo, q);
        atomicMax(s_hi, q);
      }
    }
  }
  __syncthreads();
  const int mini = *s_lo, maxi = *s_hi;
  if (q >= mini && q <= maxi) {
    ms->zeta_i[q] = ms->zeta_ii[q];
    ms->zeta_ii[q] = ms->zeta_iii[q];
  }
  if (tid == 0) {
    if (rec) rec->nsteps = nstep + 1;
    ms->lo = mini;
    ms->hi = maxi;
    ms->delta = ms->lambda;
    if (!(ms->lambda == ms->lambda)) ms->status = THR_ERR_NAN;
    if (maxi < mini || ms->it >= ms->maxcg || ms->status) ms->done = 1;
  }
}

// a batch's recorded steps folded into one affine map per shift (see msb.cu)
struct MsCoef {
  int ns, lo, hi, pad;
  double A[kMaxShift], P[kMaxShift], B[kMaxShift][kBatch], Q[kMaxShift][kBatch];
};

// destroys the cached graphs of the batched solver (context teardown)
void ms_graphs_release(thr_ctx* c);

template <class V>
int multishift_batched_dev(thr_ctx* c, const V* in, V* out, V* sf, V* ring, V* p, V* hv, V* s, int ndiagq,
                           const double* aden, const double* anum, float res, float am, int imass, int maxcg,
                           int* cg_return, int* cg_returns);

// Mixed precision: the batched FP64 solve until |r| < switch_rel |input|, then
// the base iteration (stencils, residual ring, h) in the storage type VL
// (float2: FP32; __nv_bfloat162: BF16 storage with FP32 arithmetic) while the
// shift fields out/sf stay FP64.  ring64 holds 2 kBatch FP64 fields; the VL
// ring is placed in its upper half.  low: 3 VL work fields.  *switched_at
// gets the iteration the precision changed at (0: the solve ended in FP64).
template <class VL>
int multishift_mixed_dev(thr_ctx* c, const double2* in, double2* out, double2* sf, double2* ring64, double2* p,
                         double2* hv, double2* s, VL* low, int ndiagq, const double* aden, const double* anum,
                         float res, float am, int imass, int maxcg, double switch_rel, int* cg_return,
                         int* cg_returns, int* switched_at);

// One batch (kBatch iterations on ring half `half`, recorded into rec) of the batched
// FP64 multishift as one persistent kernel on stream st (msp.cu).  THR_ERR_UNSUPPORTED
// where it does not apply (context mode, block shape, lattice size): the caller then
// launches the kernel chain.  dry: only say whether it applies.
int ms_chain_batch(thr_ctx* c, MsState* ms, MsHist* rec, double2* ring, double2* hv, double2* p, float am, int imass,
                   int half, cudaStream_t st, bool dry);

template <class V>
int multishift_dev(thr_ctx* c, const V* u_dummy, const V* in, V* out, V* sf, V* r, V* p, V* hv, V* s, int ndiagq,
                   const double* aden, const double* anum, float res, float am, int imass, int maxcg, int* cg_return,
                   int* cg_returns);

}  // namespace thr
