// overlap.h -- host entry points of overlap.cu shared with the other
// translation units (the overlap operator of measure_OWilson.F90).
#pragma once
#include "ctx.h"

namespace thr {

// prepZolo's coefficients for the context's Ls on [lmin, lmax] (host)
int zolo_coefficients(int n, double lmin, double lmax, double* out);
// the context's coefficients on the device (the reference's [0.1, 5] unless set)
int zolo_device(thr_ctx* c, const double** zc);
// congradO on device fields (measure_OWilson.F90:190-268)
int congrad_o_dev(thr_ctx* c, const double2* phi, double2* X, float res, float am, int imass, int niterc, int* itercg,
                  int* iterations);
// measure_wilsonKDDW (measure_OWilson.F90:646-673) on the current links and the
// context's random numbers; respbp is congradO's residual (params.F90:60)
int measure_ow(thr_ctx* c, float respbp, float bmass, int imass, int knoise, float* psibarpsi, float* susclsing,
               float* aviter, double* parts, int* itercg);

}  // namespace thr
