// bcg.h -- batched congrad (many right-hand sides / many lattices).
#pragma once
#include <cuda_runtime.h>

#include "batch.h"

namespace thr {

struct BcgState {
  double rr, pq, alpha, beta, target, resid, r2_true;
  int iters, inner_it, outer, done_outer, done_inner, cap, status, rounds;
  int done_at;  // inner-loop step whose residual ended the entry's inner solve (-1: none)
};

struct BcgRun {
  const BatchTable* tab = nullptr;
  int kernel = 0;
  float am = 0.f, am3 = 1.f;
  int imass = 1;
  cudaStream_t st = nullptr;
  const double2* u64 = nullptr;  // links, FP64 (packed per entry or shared)
  const void* ulow = nullptr;    // links, FP32
  int grid = 0;                  // persistent stencil grid (0 = default)
  BcgState* state = nullptr;     // [nent]
  int* skip = nullptr;           // [nent]
  double* partials = nullptr;    // >= max(total_blocks, 64 * nent)
  const double2* B = nullptr;    // right-hand sides, FP64
  double2* X = nullptr;          // solutions, FP64 (initial guesses in)
  double2 *R = nullptr, *T = nullptr, *H = nullptr;  // FP64 work
  void *r = nullptr, *p = nullptr, *h = nullptr, *q = nullptr, *e = nullptr;  // inner work (precision dependent)
  long long launches = 0;
};

// precision: THR_FP64, THR_MIXED_FP32 or THR_MIXED_BF16
int bcg_solve(BcgRun& br, int precision, float res, int max_outer, int* iters, int* outer);

}  // namespace thr
