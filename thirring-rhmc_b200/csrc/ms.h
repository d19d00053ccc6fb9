// ms.h -- multishift solver state (multishift_module.F90:43-57), device-resident.
#pragma once
#include "ctx.h"

namespace thr {

constexpr int kMaxShift = 64;

struct MsState {
  double omega, gammag, delta, alpha, lambda, omega_save;
  int it, maxcg, lo, hi, done, status, ndiagq;
  float res;
  double active_sum;  // sum over iterations of the shifts updated (for traffic accounting)
  double zeta_i[kMaxShift], zeta_ii[kMaxShift], zeta_iii[kMaxShift];
  double omegas[kMaxShift], gammas[kMaxShift], correction[kMaxShift], aden[kMaxShift];
  int flags[kMaxShift], cg_returns[kMaxShift];
};
static_assert(sizeof(MsState) <= 4096 * sizeof(double), "MsState must fit the scalar block");

int ms_prepare_state(thr_ctx* c, MsState* h, int ndiagq, const double* aden, const double* anum, float res, int maxcg);

template <class V>
int multishift_dev(thr_ctx* c, const V* u_dummy, const V* in, V* out, V* sf, V* r, V* p, V* hv, V* s, int ndiagq,
                   const double* aden, const double* anum, float res, float am, int imass, int maxcg, int* cg_return,
                   int* cg_returns);

}  // namespace thr
