// finish.cuh -- scalar steps of the solvers run by the last block of a stencil launch.
//
// A stencil launch with a reduction epilogue writes one partial per block.
// Instead of a separate one-block kernel that sums them and advances the
// solver's scalars, the last block to finish does it: every block writes its
// partial, fences and takes a ticket from an atomic counter; the block that
// draws the last ticket sums all partials in index order (so the result does
// not depend on which block finished last), runs the scalar step and resets
// the counter for the next launch.  No block ever waits for another.
#pragma once
#include "ms.h"
#include "solver.h"

namespace thr {

enum FinKind {
  FIN_NONE = 0,
  FIN_MS_ALPHA = 1,   // multishift alpha step (multishift_module.F90:104, :118-135) + step record
  FIN_MS_LAMBDA = 2,  // multishift lambda step (:138-150), record, convergence (:240-258)
  FIN_CG_ALPHA = 3,   // congrad alpha (measure_module.F90:57, :66-75)
  FIN_CG_BETA = 4     // congrad beta and stopping rule (:102-110, :120)
};

struct FinArgs {
  int kind = FIN_NONE;
  void* state = nullptr;     // MsState* or CgState*
  void* hist = nullptr;      // MsHist* (multishift)
  unsigned* counter = nullptr;
};

// called by every thread of every block after thread 0 wrote partials[bid];
// red: shared scratch of at least nthr doubles
__device__ __forceinline__ void block_finish(const FinArgs& fa, const double* partials, int nparts, double* red,
                                             int tid, int nthr) {
  __shared__ int last;
  if (tid == 0) {
    __threadfence();
    const unsigned ticket = atomicAdd(fa.counter, 1u);
    last = ticket == (unsigned)(nparts - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  // fixed-order sum of all partials
  double v = 0.0;
  for (int i = tid; i < nparts; i += nthr) v += ((volatile const double*)partials)[i];
  red[tid] = v;
  __syncthreads();
  if (tid < 32) {
    double w = 0.0;
    for (int i = tid; i < nthr; i += 32) w += red[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
    if (tid == 0) red[0] = w;
  }
  __syncthreads();
  const double total = red[0];
  if (fa.kind == FIN_MS_ALPHA) {
    MsState* ms = (MsState*)fa.state;
    MsHist* hist = (MsHist*)fa.hist;
    if (tid == 0) {
      ms_alpha_scalar(ms, total);
      hist->lo[hist->nsteps] = ms->lo;
      hist->hi[hist->nsteps] = ms->hi;
    }
    __syncthreads();
    for (int k = ms->lo + tid; k <= ms->hi; k += nthr) {
      ms_alpha_shift(ms, k);
      hist->om[hist->nsteps][k] = ms->omegas[k];
      hist->ze[hist->nsteps][k] = ms->zeta_iii[k];
    }
  } else if (fa.kind == FIN_MS_LAMBDA) {
    MsState* ms = (MsState*)fa.state;
    MsHist* hist = (MsHist*)fa.hist;
    if (tid == 0) ms_lambda_scalar(ms, total);
    __syncthreads();
    for (int k = ms->lo + tid; k <= ms->hi; k += nthr) {
      ms_lambda_shift(ms, k);
      hist->ga[hist->nsteps][k] = ms->gammas[k];
    }
    __syncthreads();
    if (tid == 0) {
      hist->nsteps += 1;
      ms_converge_step(ms);
    }
  } else if (fa.kind == FIN_CG_ALPHA) {
    CgState* cs = (CgState*)fa.state;
    if (tid == 0) {
      cs->nx += 1;
      cs->itercg += 1;
      if (cs->nx != 1) cs->alpha = cs->alphan / total;
      cs->nalpha = -cs->alpha;
    }
  } else if (fa.kind == FIN_CG_BETA) {
    CgState* cs = (CgState*)fa.state;
    if (tid == 0) {
      const double betacgn = total;
      double betacg = betacgn / cs->betacgd;
      cs->betacgd = betacgn;
      cs->alphan = betacgn;
      if (cs->nx == 1) betacg = 0.0;
      cs->betacg = betacg;
      cs->betacgn = betacgn;
      if (!(betacgn == betacgn)) {
        cs->status = THR_ERR_NAN;
        cs->pending_done = 1;
      }
      if (betacgn < cs->resid) cs->pending_done = 1;
      else if (cs->nx >= cs->niterc) {
        cs->pending_done = 1;
        cs->capped = 1;
      }
    }
  }
  if (tid == 0) *fa.counter = 0u;
}

}  // namespace thr
