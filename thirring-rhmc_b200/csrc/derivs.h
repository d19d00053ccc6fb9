// derivs.h -- fermion force launcher (derivs_module.F90:8-410).
#pragma once
#include "ctx.h"

namespace thr {
// dS[mu][site] += force contribution of (R, X2) with coefficient anum
int launch_derivs(thr_ctx* c, double* dS, const double2* R, const double2* X2, double anum, int iflag, float am,
                  int imass);
}  // namespace thr
