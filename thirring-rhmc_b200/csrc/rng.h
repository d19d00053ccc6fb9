// rng.h -- random-number state (site_random.f90 / random.f90) held by a context.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

struct thr_ctx;

namespace thr {

struct Rng {
  bool ready = false;
  bool site = true;           // site_random.f90 streams (device) vs random.f90 (host)
  void* dev_streams = nullptr;  // per-site {S, y, idum}
  void* dev_tables = nullptr;   // per-site 97-entry shuffle tables, [97][V3]
  uint64_t hS = 2868876ULL * 16777216ULL + 16651885ULL;  // DATA DS (random.f90:20)
  float hv[97] = {};
  float hy = 0.0f;
  int hidum = -1;
  float hscratch = 0.0f;
  int ensure(thr_ctx* c);
  void release();
};

int rng_init(thr_ctx* c, double seed, int site_mode);
int rng_gauss_dev(thr_ctx* c, float scale, float* ps);  // ps[2][V3] device, storage order
int rng_phi_draw(thr_ctx* c, double2* R);                // evolution.F90:40-51
int rng_pp_draw(thr_ctx* c, float* pp);                  // evolution.F90:93-109, pp[3][V3]
int rng_rano_site(thr_ctx* c, int ix, int iy, int it, float* dout, float* hout);
void rng_natural_to_storage(thr_ctx* c, float* out, const float* in, int ncomp);

}  // namespace thr
