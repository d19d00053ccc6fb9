// md.h -- device-resident RHMC layer (force, hamilton, MD, trajectory).
#pragma once
#include "ctx.h"

namespace thr {

struct MdFields {
  double2 *Phi, *X2, *Xr, *R;  // spinors
  float *theta, *thetat, *pp;  // [3][V3] single precision
  double* dS;                  // gforce::dSdpi [3][V3]
};

int md_fields(thr_ctx* c, MdFields* f);
int force_dev(thr_ctx* c, MdFields* f, const float* theta, float res1, float am, int imass);
int hamilton_dev(thr_ctx* c, MdFields* f, const float* theta, const float* pp, float res2, float am, int imass,
                 double* h, double* hg, double* hp, double* s);
int initialise_phi_dev(thr_ctx* c, MdFields* f, float am, int imass);
int evolve_dev(thr_ctx* c, MdFields* f, int iterl, float dt, float res, float am, int imass, int fixed_steps,
               int* itot);
int trajectory_dev(thr_ctx* c, MdFields* f, int iterl, float dt, float am, int imass, int fixed_steps,
                   thr_traj_result* out);
// destroys the cached MD step graph (context teardown)
void md_graph_release(thr_ctx* c);

}  // namespace thr
