// qmr.h -- qmrherm and multishift on device fields.
#pragma once
#include "ctx.h"

namespace thr {
int multishift_into(thr_ctx* c, const double2* Phi, double2* x1, int nq, const double* aden, const double* anum,
                    float res, float am, int imass, int maxcg, int sp, int* itercg, int* cg_returns);
int qmrherm_dev(thr_ctx* c, const double2* Phi, double2* x, float res, int* itercg, float am, int imass,
                const double* anum, const double* aden, int nq, int iflag, int use_sp, int* cg_returns, double* dS,
                int max_iters);
}  // namespace thr
