// solver.h -- device-resident solver state shared by the solver units.
#pragma once
#include "ctx.h"

namespace thr {

// congrad scalars (measure_module.F90:29-31), kept in device memory
struct CgState {
  double alpha, alphan, betacg, betacgd, betacgn, resid, nalpha;  // nalpha = -alpha for the fused r update
  int nx, itercg, niterc, done, pending_done, capped, status, chunks, max_chunks, pad;
};

template <class S>
inline int launch_dslash_guarded(thr_ctx* c, bool dag, S* out, const S* in, const typename Sto<S>::C* u, float am,
                                 int imass, const int* skip) {
  return launch_dslash<S>(c->g, c->p.kernel, dag, out, in, u, am, imass, c->p.am3, c->st, skip);
}

int congrad_dev(thr_ctx* c, const double2* Phi, double2* X, float res, float am, int imass, int niterc, int* itercg,
                int* iterations);
// destroys the cached congrad graph (context teardown)
void cg_graph_release(thr_ctx* c);

}  // namespace thr
