// bcg_abi.cu -- C ABI of the batched congrad: many right-hand sides on a
// context's lattice (thr_congrad_multi*) and many independent lattices of
// uneven sizes packed together (thr_pack_*).
#include <algorithm>
#include <cstring>
#include <vector>

#include "bcg.h"
#include "ctx.h"

namespace thr {

namespace {
__global__ void k_links32(float2* d, const double2* s, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    d[i] = make_float2((float)s[i].x, (float)s[i].y);
}
}  // namespace

// device buffers of one batched solve
struct BatchBufs {
  BatchTable tab;
  BcgState* state = nullptr;
  int* skip = nullptr;
  double* partials = nullptr;
  double2 *B = nullptr, *X = nullptr, *R = nullptr, *T = nullptr, *H = nullptr;
  void *r = nullptr, *p = nullptr, *h = nullptr, *q = nullptr, *e = nullptr;
  double2* u64 = nullptr;
  float2* u32 = nullptr;
  void* stage = nullptr;
  size_t stage_bytes = 0;
  ~BatchBufs() { release(); }
  void release() {
    for (void* ptr : {(void*)state, (void*)skip, (void*)partials, (void*)B, (void*)X, (void*)R, (void*)T, (void*)H, r,
                      p, h, q, e, (void*)u64, (void*)u32, stage})
      cudaFree(ptr);
    state = nullptr; skip = nullptr; partials = nullptr; B = X = R = T = H = nullptr;
    r = p = h = q = e = nullptr; u64 = nullptr; u32 = nullptr; stage = nullptr;
  }
  int alloc(bool own_links, size_t stage_b) {
    const size_t n = (size_t)tab.total_elems, ne = (size_t)tab.nent;
    const size_t nparts = std::max((size_t)tab.total_blocks, 64 * ne) + 64;
    bool ok = cudaMalloc(&state, sizeof(BcgState) * ne) == cudaSuccess && cudaMalloc(&skip, sizeof(int) * ne) == cudaSuccess &&
              cudaMalloc(&partials, sizeof(double) * nparts) == cudaSuccess;
    for (double2** f : {&B, &X, &R, &T, &H}) ok = ok && cudaMalloc(f, n * sizeof(double2)) == cudaSuccess;
    // the inner vectors are sized for FP64 so any precision fits
    for (void** f : {&r, &p, &h, &q, &e}) ok = ok && cudaMalloc(f, n * sizeof(double2)) == cudaSuccess;
    if (own_links) {
      ok = ok && cudaMalloc(&u64, (size_t)tab.total_links * sizeof(double2)) == cudaSuccess &&
           cudaMalloc(&u32, (size_t)tab.total_links * sizeof(float2)) == cudaSuccess;
    }
    if (stage_b) {
      ok = ok && cudaMalloc(&stage, stage_b) == cudaSuccess;
      stage_bytes = stage_b;
    }
    return ok ? THR_OK : THR_ERR_NOMEM;
  }
};

}  // namespace thr

using namespace thr;

struct thr_pack {
  int dev = 0;
  cudaStream_t st = nullptr;
  std::vector<thr_params> p;
  std::vector<Geom> geoms;
  BatchBufs bb;
  bool links_ready = false;
  long long launches = 0;
};

namespace {
Geom geom_of(const thr_params& p) {
  return geom_make(p.lx, p.ly, p.lt, p.ls, p.layout);
}
size_t nf5_of(const Geom& g) { return (size_t)(g.ls + 2) * (g.lx + 2) * (g.ly + 2) * (g.lt + 2) * 4; }

int run_batch(BatchBufs& bb, cudaStream_t st, int kernel, float am3, const double2* u64, const void* u32, float res,
              float am, int imass, int precision, int* itercg, int* outer, long long* launches) {
  if (precision != THR_FP64 && precision != THR_MIXED_FP32 && precision != THR_MIXED_BF16) return THR_ERR_BADARG;
  BcgRun br;
  br.tab = &bb.tab;
  br.kernel = kernel;
  br.am = am;
  br.am3 = am3;
  br.imass = imass;
  br.st = st;
  br.u64 = u64;
  br.ulow = u32;
  br.state = bb.state;
  br.skip = bb.skip;
  br.partials = bb.partials;
  br.B = bb.B;
  br.X = bb.X;
  br.R = bb.R;
  br.T = bb.T;
  br.H = bb.H;
  br.r = bb.r;
  br.p = bb.p;
  br.h = bb.h;
  br.q = bb.q;
  br.e = bb.e;
  const int rc = bcg_solve(br, precision, res, 64, itercg, outer);
  if (launches) *launches += br.launches;
  return rc;
}
}  // namespace

extern "C" {

// ---------------------------------------------------------------- right-hand sides on one lattice
int thr_congrad_multi_dev(thr_ctx* c, const void* Phi, void* X, int nrhs, float res, float am, int imass,
                          int precision, int* itercg, int* outer) {
  if (!c || !Phi || !X || nrhs < 1) return THR_ERR_BADARG;
  if (imass != 1 && imass != 3 && imass != 5) return THR_ERR_BADARG;
  if (!c->links_ok) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  BatchBufs bb;
  std::vector<Geom> gs(nrhs, c->g);
  THR_TRY(bb.tab.build(gs, true, c->st));
  THR_TRY(bb.alloc(false, 0));
  const size_t bytes = (size_t)bb.tab.total_elems * sizeof(double2);
  THR_CUDA(cudaMemcpyAsync(bb.B, Phi, bytes, cudaMemcpyDeviceToDevice, c->st));
  THR_CUDA(cudaMemcpyAsync(bb.X, X, bytes, cudaMemcpyDeviceToDevice, c->st));
  int rc = run_batch(bb, c->st, c->p.kernel, c->p.am3, c->u64, c->u32, res, am, imass, precision, itercg, outer,
                     nullptr);
  if (rc != THR_OK && rc != THR_ERR_MAXITER) return rc;
  THR_CUDA(cudaMemcpyAsync(X, bb.X, bytes, cudaMemcpyDeviceToDevice, c->st));
  THR_CUDA(cudaStreamSynchronize(c->st));
  return rc;
}

int thr_congrad_multi(thr_ctx* c, const double* Phi, double* X, int nrhs, float res, float am, int imass,
                      int precision, int* itercg, int* outer) {
  if (!c || !Phi || !X || nrhs < 1) return THR_ERR_BADARG;
  if (imass != 1 && imass != 3 && imass != 5) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  THR_TRY(c->use_links(nullptr));
  BatchBufs bb;
  std::vector<Geom> gs(nrhs, c->g);
  THR_TRY(bb.tab.build(gs, true, c->st));
  THR_TRY(bb.alloc(false, 0));
  const size_t n = c->n4(), nf = c->nf5();
  for (int k = 0; k < nrhs; k++) {
    THR_TRY(c->upload_spinor(bb.B + k * n, Phi + 2 * nf * k));
    THR_TRY(c->upload_spinor(bb.X + k * n, X + 2 * nf * k));
  }
  int rc = run_batch(bb, c->st, c->p.kernel, c->p.am3, c->u64, c->u32, res, am, imass, precision, itercg, outer,
                     nullptr);
  if (rc != THR_OK && rc != THR_ERR_MAXITER) return rc;
  for (int k = 0; k < nrhs; k++) THR_TRY(c->download_spinor(X + 2 * nf * k, bb.X + k * n));
  int rs = c->sync();
  return rs ? rs : rc;
}

// ---------------------------------------------------------------- packed lattices
int thr_pack_create(int n, const thr_params* p, int device, thr_pack** out) {
  if (n < 1 || !p || !out) return THR_ERR_BADARG;
  *out = nullptr;
  thr_pack* k = new thr_pack();
  k->dev = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&k->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete k;
    return THR_ERR_CUDA;
  }
  size_t stage = 0;
  for (int i = 0; i < n; i++) {
    if (p[i].lx < 2 || p[i].ly < 2 || p[i].lt < 2 || p[i].ls < 1 || p[i].ls > 256) {
      thr_pack_destroy(k);
      return THR_ERR_BADSHAPE;
    }
    if (p[i].kernel != p[0].kernel) {
      thr_pack_destroy(k);
      return THR_ERR_BADARG;  // one operator kind per pack
    }
    k->p.push_back(p[i]);
    k->geoms.push_back(geom_of(p[i]));
    stage = std::max(stage, nf5_of(k->geoms.back()) * sizeof(double2));
  }
  int rc = k->bb.tab.build(k->geoms, false, k->st);
  if (!rc) rc = k->bb.alloc(true, stage);
  if (rc) {
    thr_pack_destroy(k);
    return rc;
  }
  *out = k;
  return THR_OK;
}

int thr_pack_destroy(thr_pack* k) {
  if (!k) return THR_OK;
  cudaSetDevice(k->dev);
  if (k->st) cudaStreamSynchronize(k->st);
  k->bb.release();
  if (k->st) cudaStreamDestroy(k->st);
  delete k;
  return THR_OK;
}

// links u (Fortran links layout), right-hand side Phi and initial guess X (Fortran spinors) of lattice i
int thr_pack_upload(thr_pack* k, int i, const double* u, const double* Phi, const double* X) {
  if (!k || i < 0 || i >= (int)k->geoms.size() || !u || !Phi || !X) return THR_ERR_BADARG;
  cudaSetDevice(k->dev);
  const Geom& g = k->geoms[i];
  const BatchEntry& E = k->bb.tab.host[i];
  double2* st = (double2*)k->bb.stage;
  const size_t nl = (size_t)(g.lx + 2) * (g.ly + 2) * (g.lt + 2) * 3;
  THR_CUDA(cudaMemcpyAsync(st, u, nl * sizeof(double2), cudaMemcpyHostToDevice, k->st));
  from_fortran_links(g, k->bb.u64 + E.uoff, st, k->st);
  k_links32<<<64, 256, 0, k->st>>>(k->bb.u32 + E.uoff, k->bb.u64 + E.uoff, (size_t)g.v3 * 3);
  THR_CUDA(cudaMemcpyAsync(st, Phi, nf5_of(g) * sizeof(double2), cudaMemcpyHostToDevice, k->st));
  from_fortran_spinor<double2>(g, k->bb.B + E.off, st, k->st);
  THR_CUDA(cudaMemcpyAsync(st, X, nf5_of(g) * sizeof(double2), cudaMemcpyHostToDevice, k->st));
  from_fortran_spinor<double2>(g, k->bb.X + E.off, st, k->st);
  THR_CUDA(cudaStreamSynchronize(k->st));
  return THR_OK;
}

int thr_pack_congrad(thr_pack* k, float res, float am, int imass, int precision, int* itercg, int* outer) {
  if (!k) return THR_ERR_BADARG;
  if (imass != 1 && imass != 3 && imass != 5) return THR_ERR_BADARG;
  cudaSetDevice(k->dev);
  const thr_params& p0 = k->p[0];
  return run_batch(k->bb, k->st, p0.kernel, p0.am3, k->bb.u64, k->bb.u32, res, am, imass, precision, itercg, outer,
                   &k->launches);
}

int thr_pack_download(thr_pack* k, int i, double* X) {
  if (!k || i < 0 || i >= (int)k->geoms.size() || !X) return THR_ERR_BADARG;
  cudaSetDevice(k->dev);
  const Geom& g = k->geoms[i];
  const BatchEntry& E = k->bb.tab.host[i];
  to_fortran_spinor(g, (double2*)k->bb.stage, k->bb.X + E.off, k->st);
  THR_CUDA(cudaMemcpyAsync(X, k->bb.stage, nf5_of(g) * sizeof(double2), cudaMemcpyDeviceToHost, k->st));
  THR_CUDA(cudaStreamSynchronize(k->st));
  return THR_OK;
}

int thr_pack_zero_x(thr_pack* k) {
  if (!k) return THR_ERR_BADARG;
  cudaSetDevice(k->dev);
  THR_CUDA(cudaMemsetAsync(k->bb.X, 0, (size_t)k->bb.tab.total_elems * sizeof(double2), k->st));
  THR_CUDA(cudaStreamSynchronize(k->st));
  return THR_OK;
}

int thr_pack_get_stream(thr_pack* k, void** stream) {
  if (!k || !stream) return THR_ERR_BADARG;
  *stream = (void*)k->st;
  return THR_OK;
}

}  // extern "C"
