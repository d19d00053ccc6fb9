// ctx.cu -- context lifetime, host<->device transfers, links, and the
// dirac.F90 / gauge.F90 entry points of the C ABI.
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <type_traits>

#include "ctx.h"
#include "md.h"
#include "ms.h"
#include "solver.h"

using namespace thr;

int thr_ctx::ensure_w64(int count) {
  if (md_capture && (int)w64.size() < count) return THR_ERR_BADSHAPE;  // no allocation inside a capture
  while ((int)w64.size() < count) {
    buf_gen++;
    double2* p = nullptr;
    if (cudaMalloc(&p, n4() * sizeof(double2)) != cudaSuccess) return THR_ERR_NOMEM;
    cudaMemsetAsync(p, 0, n4() * sizeof(double2), st);
    w64.push_back(p);
  }
  return THR_OK;
}

int thr_ctx::buffer(int id, size_t bytes, void** out) {
  if (id < 0 || id >= B_COUNT) return THR_ERR_BADARG;
  if (buf_bytes[id] < bytes) {
    if (md_capture) return THR_ERR_BADSHAPE;  // no allocation inside a capture
    buf_gen++;
    cudaStreamSynchronize(st);
    cudaFree(bufs[id]);
    bufs[id] = nullptr;
    buf_bytes[id] = 0;
    if (cudaMalloc(&bufs[id], bytes) != cudaSuccess) return THR_ERR_NOMEM;
    buf_bytes[id] = bytes;
    cudaMemsetAsync(bufs[id], 0, bytes, st);
    if (id == B_PHI0) phi0_valid = false;
  }
  *out = bufs[id];
  return THR_OK;
}

int thr_ctx::prof_begin(int kind, double bytes, long long tag, cudaStream_t on) {
  if (!prof_on) return -1;
  if (prof_seen[kind]++ % prof_stride) return -1;
  const int idx = (int)prof_kind.size();
  if (2 * idx + 2 > (int)prof_ev.size()) {
    for (int k = 0; k < 256; k++) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      prof_ev.push_back(e);
    }
  }
  prof_kind.push_back(kind);
  prof_bytes.push_back(bytes);
  prof_tag.push_back(tag);
  cudaEventRecord(prof_ev[2 * idx], on ? on : st);
  return idx;
}
void thr_ctx::prof_end(int idx, cudaStream_t on) {
  if (idx >= 0) cudaEventRecord(prof_ev[2 * idx + 1], on ? on : st);
}
void thr_ctx::prof_set_bytes(int idx, double bytes) {
  if (idx >= 0 && idx < (int)prof_bytes.size()) prof_bytes[idx] = bytes;
}
void thr_ctx::prof_trim(size_t first, long long iters) {
  for (size_t i = first; i < prof_kind.size(); i++)
    if (prof_tag[i] >= iters) prof_kind[i] = -1;
}

int thr_ctx::upload_spinor(double2* dst, const double* host) {
  THR_CUDA(cudaMemcpyAsync(stage, host, nf5() * sizeof(double2), cudaMemcpyHostToDevice, st));
  from_fortran_spinor<double2>(g, dst, stage, st);
  return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
}

int thr_ctx::download_spinor(double* host, const double2* src) {
  to_fortran_spinor(g, stage, src, st);
  THR_CUDA(cudaMemcpyAsync(host, stage, nf5() * sizeof(double2), cudaMemcpyDeviceToHost, st));
  return THR_OK;
}

namespace {
__global__ void k_links_f32(float2* d, const double2* s, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    d[i] = make_float2((float)s[i].x, (float)s[i].y);  // u = cmplx(udp): multishift_module.F90:351
}
// coef: gauge.F90:27-32
__global__ void k_coef(double2* u, const float* theta, Geom g, int ibound) {
  int n = g.v3 * 3;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int site = i % g.v3, mu = i / g.v3;
    int x, y, t;
    site_coords(g, site, x, y, t);
    float re = 1.0f + 0.0f, im = theta[i];
    double2 v = make_double2((double)re, (double)im);
    if (ibound == -1 && mu == 2 && t == g.lt - 1) v = make_double2(-v.x, -v.y);
    u[i] = v;
  }
}
}  // namespace

int thr_ctx::use_links(const double* u_host) {
  if (u_host) {
    THR_CUDA(cudaMemcpyAsync(stage, u_host, nfl() * sizeof(double2), cudaMemcpyHostToDevice, st));
    from_fortran_links(g, u64, stage, st);
    links_ok = true;
  }
  if (!links_ok) return THR_ERR_BADARG;
  k_links_f32<<<(g.v3 * 3 + 255) / 256, 256, 0, st>>>(u32, u64, g.v3 * 3);
  return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
}

// u = coef(theta) from a device theta[3][V3] (storage order); refreshes the FP32 copy
int thr_ctx::coef_dev(const float* theta_dev) {
  const size_t n3 = (size_t)g.v3 * 3;
  k_coef<<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(u64, theta_dev, g, p.ibound);
  links_ok = true;
  return use_links(nullptr);
}

int thr_ctx::sync() {
  THR_CUDA(cudaStreamSynchronize(st));
  return THR_OK;
}

// ---------------------------------------------------------------- C ABI
extern "C" {

const char* thr_status_string(int s) {
  switch (s) {
    case THR_OK: return "ok";
    case THR_ERR_BADARG: return "bad argument";
    case THR_ERR_BADSHAPE: return "bad shape";
    case THR_ERR_MAXITER: return "iteration cap reached";
    case THR_ERR_NAN: return "non-finite value";
    case THR_ERR_CUDA: return "CUDA error";
    case THR_ERR_NOMEM: return "out of device memory";
    case THR_ERR_UNSUPPORTED: return "unsupported option";
    case THR_ERR_TIMEOUT: return "device-side wait timed out";
    default: return "unknown status";
  }
}

int thr_create(const thr_params* p, thr_ctx** out) {
  if (!p || !out) return THR_ERR_BADARG;
  *out = nullptr;
  if (p->lx < 2 || p->ly < 2 || p->lt < 2 || p->ls < 1 || p->ls > 1024) return THR_ERR_BADSHAPE;
  if (p->kernel != 0 && p->kernel != 1) return THR_ERR_BADARG;
  if (p->layout == 1 && (p->lx % 2 != 0)) return THR_ERR_BADSHAPE;
  thr_ctx* c = new thr_ctx();
  c->p = *p;
  if (c->p.ndiag <= 0) c->p.ndiag = 25;
  c->g = thr::geom_make(p->lx, p->ly, p->lt, p->ls, p->layout);
  c->dev = p->device;
  {
    const char* e = std::getenv("THR_REVERSE");
    if (e && (e[0] == '0' || e[0] == '1')) c->rev_sweep = e[0] - '0';
    e = std::getenv("THR_OVERLAP");
    if (e && e[0] == '0') c->overlap_flush = 0;
    // THR_GRAPHS=0: solver loops launched from the host (profilers cannot look inside
    // graphs with conditional nodes)
    e = std::getenv("THR_GRAPHS");
    if (e && e[0] == '0') c->use_graphs = false;
    e = std::getenv("THR_MD_GRAPH");
    if (e && e[0] == '0') c->use_md_graph = false;
    e = std::getenv("THR_PDL");
    if (e && e[0] == '0') c->use_pdl = false;
    e = std::getenv("THR_CHAIN");
    if (e && (e[0] == '0' || e[0] == '1' || e[0] == '2') && e[1] == 0) c->chain_mode = e[0] - '0';
  }
  int rc = THR_OK;
  if (cudaSetDevice(c->dev) != cudaSuccess) rc = THR_ERR_CUDA;
  int prio_lo = 0, prio_hi = 0;  // numerically: lo >= hi
  if (!rc && cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi) != cudaSuccess) rc = THR_ERR_CUDA;
  if (!rc && cudaStreamCreateWithPriority(&c->st, cudaStreamNonBlocking, prio_hi) != cudaSuccess) rc = THR_ERR_CUDA;
  if (!rc && cudaStreamCreateWithPriority(&c->st2, cudaStreamNonBlocking, prio_lo) != cudaSuccess) rc = THR_ERR_CUDA;
  if (!rc && cudaStreamCreateWithPriority(&c->st3, cudaStreamNonBlocking, prio_hi) != cudaSuccess) rc = THR_ERR_CUDA;
  if (!rc && (cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess)) rc = THR_ERR_CUDA;
  for (int i = 0; i < 2 && !rc; i++)
    if (cudaEventCreateWithFlags(&c->ev_fork[i], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_join[i], cudaEventDisableTiming) != cudaSuccess)
      rc = THR_ERR_CUDA;
  if (!rc && cudaMalloc(&c->u64, (size_t)c->g.v3 * 3 * sizeof(double2)) != cudaSuccess) rc = THR_ERR_NOMEM;
  if (!rc && cudaMalloc(&c->u32, (size_t)c->g.v3 * 3 * sizeof(float2)) != cudaSuccess) rc = THR_ERR_NOMEM;
  c->stage_elems = c->nf5();
  if (!rc && cudaMalloc(&c->stage, c->stage_elems * sizeof(double2)) != cudaSuccess) rc = THR_ERR_NOMEM;
  // per-block partial sums: the stencil epilogue writes one per block of its grid
  const size_t nparts = std::max<size_t>((size_t)kMaxPartials * 8, (size_t)std::max(stencil_grid(c->g, 0), stencil_grid(c->g, 1)) + 1024);
  if (!rc && cudaMalloc(&c->partials, nparts * sizeof(double)) != cudaSuccess) rc = THR_ERR_NOMEM;
  c->nparts = nparts;
  if (!rc && cudaMalloc(&c->dscal, 4096 * sizeof(double)) != cudaSuccess) rc = THR_ERR_NOMEM;
  if (!rc && cudaMalloc(&c->iscal, 1024 * sizeof(int)) != cudaSuccess) rc = THR_ERR_NOMEM;
  if (!rc && cudaMallocHost(&c->hscal, 4096 * sizeof(double)) != cudaSuccess) rc = THR_ERR_NOMEM;
  if (!rc && cudaMallocHost(&c->hiscal, 1024 * sizeof(int)) != cudaSuccess) rc = THR_ERR_NOMEM;
  if (!rc && cudaMallocHost(&c->ms_tmpl, kMsTemplates * sizeof(MsState)) != cudaSuccess) rc = THR_ERR_NOMEM;
  if (rc) {
    thr_destroy(c);
    return rc;
  }
  cudaMemsetAsync(c->dscal, 0, 4096 * sizeof(double), c->st);
  cudaMemsetAsync(c->iscal, 0, 1024 * sizeof(int), c->st);
  *out = c;
  return THR_OK;
}

int thr_destroy(thr_ctx* c) {
  if (!c) return THR_OK;
  cudaSetDevice(c->dev);
  if (c->st) cudaStreamSynchronize(c->st);
  if (c->st2) cudaStreamSynchronize(c->st2);
  ms_graphs_release(c);
  cg_graph_release(c);
  md_graph_release(c);
  for (auto p : c->w64) cudaFree(p);
  for (auto e : c->prof_ev) cudaEventDestroy(e);
  for (int i = 0; i < thr_ctx::B_COUNT; i++) cudaFree(c->bufs[i]);
  c->rng.release();
  cudaFree(c->u64);
  cudaFree(c->u32);
  cudaFree(c->stage);
  cudaFree(c->stage2);
  cudaFree(c->partials);
  cudaFree(c->zolo_dev);
  cudaFree(c->dscal);
  cudaFree(c->iscal);
  if (c->hscal) cudaFreeHost(c->hscal);
  if (c->hiscal) cudaFreeHost(c->hiscal);
  if (c->ms_tmpl) cudaFreeHost(c->ms_tmpl);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  for (int i = 0; i < 2; i++) {
    if (c->ev_fork[i]) cudaEventDestroy(c->ev_fork[i]);
    if (c->ev_join[i]) cudaEventDestroy(c->ev_join[i]);
  }
  if (c->st2) cudaStreamDestroy(c->st2);
  if (c->st3) cudaStreamDestroy(c->st3);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
  return THR_OK;
}

int thr_set_am3(thr_ctx* c, float am3) {
  if (!c) return THR_ERR_BADARG;
  c->p.am3 = am3;
  return THR_OK;
}
int thr_set_beta(thr_ctx* c, float beta) {
  if (!c) return THR_ERR_BADARG;
  c->p.beta = beta;
  return THR_OK;
}

int thr_host_register(void* ptr, unsigned long long bytes) {
  if (!ptr) return THR_ERR_BADARG;
  return cudaHostRegister(ptr, (size_t)bytes, cudaHostRegisterDefault) == cudaSuccess ? THR_OK : THR_ERR_CUDA;
}
int thr_host_unregister(void* ptr) {
  if (!ptr) return THR_ERR_BADARG;
  return cudaHostUnregister(ptr) == cudaSuccess ? THR_OK : THR_ERR_CUDA;
}

int thr_set_links(thr_ctx* c, const double* u) {
  if (!c || !u) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  THR_TRY(c->use_links(u));
  return c->sync();
}

int thr_coef(thr_ctx* c, double* u, const float* theta) {
  if (!c || !theta) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  float* th = reinterpret_cast<float*>(c->stage2 ? c->stage2 : c->stage);
  // theta (Lx,Ly,Lt,3) -> staging (raw) -> device order in the second half of stage
  size_t n3 = (size_t)c->g.v3 * 3;
  float* thd = th + n3;
  THR_CUDA(cudaMemcpyAsync(th, theta, n3 * sizeof(float), cudaMemcpyHostToDevice, c->st));
  from_fortran_f3(c->g, thd, th, c->st);
  k_coef<<<(unsigned)((n3 + 255) / 256), 256, 0, c->st>>>(c->u64, thd, c->g, c->p.ibound);
  c->links_ok = true;
  THR_TRY(c->use_links(nullptr));
  if (u) {
    to_fortran_links(c->g, c->stage, c->u64, c->st);
    THR_CUDA(cudaMemcpyAsync(u, c->stage, c->nfl() * sizeof(double2), cudaMemcpyDeviceToHost, c->st));
  }
  return c->sync();
}

static int dslash_common(thr_ctx* c, double* Phi, const double* R, const double* u, float am, int imass, bool dag) {
  if (!c || !Phi || !R) return THR_ERR_BADARG;
  if (imass != 1 && imass != 3 && imass != 5) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  THR_TRY(c->ensure_w64(2));
  THR_TRY(c->use_links(u));
  THR_TRY(c->upload_spinor(c->w64[0], R));
  THR_TRY(launch_dslash<double2>(c->g, c->p.kernel, dag, c->w64[1], c->w64[0], c->u64, am, imass, c->p.am3, c->st));
  THR_TRY(c->download_spinor(Phi, c->w64[1]));
  return c->sync();
}

int thr_dslash(thr_ctx* c, double* Phi, const double* R, const double* u, float am, int imass) {
  return dslash_common(c, Phi, R, u, am, imass, false);
}
int thr_dslashd(thr_ctx* c, double* Phi, const double* R, const double* u, float am, int imass) {
  return dslash_common(c, Phi, R, u, am, imass, true);
}

}  // extern "C"

// ---------------------------------------------------------------- device fields
static size_t prec_bytes(int precision) {
  switch (precision) {
    case THR_FP64: return sizeof(double2);
    case THR_FP32_REF:
    case THR_MIXED_FP32: return sizeof(float2);
    case THR_MIXED_BF16: return sizeof(__nv_bfloat162);
    default: return 0;
  }
}

extern "C" {

int thr_field_create(thr_ctx* c, int precision, void** f) {
  if (!c || !f || !prec_bytes(precision)) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  void* p = nullptr;
  if (cudaMalloc(&p, c->n4() * prec_bytes(precision)) != cudaSuccess) return THR_ERR_NOMEM;
  THR_CUDA(cudaMemsetAsync(p, 0, c->n4() * prec_bytes(precision), c->st));
  *f = p;
  return THR_OK;
}

int thr_field_destroy(thr_ctx* c, void* f) {
  if (!c) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  cudaStreamSynchronize(c->st);
  return cudaFree(f) == cudaSuccess ? THR_OK : THR_ERR_CUDA;
}

int thr_field_upload(thr_ctx* c, void* f, int precision, const double* host) {
  if (!c || !f || !host || !prec_bytes(precision)) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  THR_CUDA(cudaMemcpyAsync(c->stage, host, c->nf5() * sizeof(double2), cudaMemcpyHostToDevice, c->st));
  if (precision == THR_FP64) from_fortran_spinor<double2>(c->g, (double2*)f, c->stage, c->st);
  else if (precision == THR_MIXED_BF16) {
    THR_TRY(c->ensure_w64(1));
    from_fortran_spinor<double2>(c->g, c->w64[0], c->stage, c->st);
    convert<__nv_bfloat162, double2>((__nv_bfloat162*)f, c->w64[0], c->n4(), c->st);
  } else from_fortran_spinor<float2>(c->g, (float2*)f, c->stage, c->st);
  return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
}

int thr_field_download(thr_ctx* c, double* host, const void* f, int precision) {
  if (!c || !f || !host || !prec_bytes(precision)) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  const double2* src = (const double2*)f;
  if (precision != THR_FP64) {
    THR_TRY(c->ensure_w64(1));
    if (precision == THR_MIXED_BF16) convert<double2, __nv_bfloat162>(c->w64[0], (const __nv_bfloat162*)f, c->n4(), c->st);
    else convert<double2, float2>(c->w64[0], (const float2*)f, c->n4(), c->st);
    src = c->w64[0];
  }
  THR_TRY(c->download_spinor(host, src));
  return c->sync();
}

int thr_dslash_dev(thr_ctx* c, void* out, const void* in, int precision, float am, int imass, int dag) {
  if (!c || !out || !in) return THR_ERR_BADARG;
  if (imass != 1 && imass != 3 && imass != 5) return THR_ERR_BADARG;
  if (!c->links_ok) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  switch (precision) {
    case THR_FP64:
      return launch_dslash<double2>(c->g, c->p.kernel, dag != 0, (double2*)out, (const double2*)in, c->u64, am, imass,
                                    c->p.am3, c->st);
    case THR_FP32_REF:
    case THR_MIXED_FP32:
      return launch_dslash<float2>(c->g, c->p.kernel, dag != 0, (float2*)out, (const float2*)in, c->u32, am, imass,
                                   c->p.am3, c->st);
    case THR_MIXED_BF16:
      return launch_dslash<__nv_bfloat162>(c->g, c->p.kernel, dag != 0, (__nv_bfloat162*)out,
                                           (const __nv_bfloat162*)in, c->u32, am, imass, c->p.am3, c->st);
    default: return THR_ERR_BADARG;
  }
}

// the solvers' fused stencil epilogues on device fields; the coefficient goes
// through a device scalar (the kernels read it from memory, as in the solvers)
int thr_dslash_fused_dev(thr_ctx* c, void* out, const void* in, const void* aux, double coef, int precision,
                         float am, int imass, int dag, int mode, double* norm2) {
  if (!c || !out || !in) return THR_ERR_BADARG;
  if (imass != 1 && imass != 3 && imass != 5) return THR_ERR_BADARG;
  if (mode != 0 && mode != 1 && mode != 3) return THR_ERR_BADARG;
  if (mode != 0 && (!aux || aux == out || aux == in)) return THR_ERR_BADARG;
  if (mode == 3 && !norm2) return THR_ERR_BADARG;
  if (mode == 1 && !norm2) return THR_ERR_BADARG;
  if (!c->links_ok) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  double* dcoef = c->dscal + kScalFusedCoef;
  double* dsum = c->dscal + kScalFusedSum;
  THR_CUDA(cudaMemcpyAsync(dcoef, &coef, sizeof(double), cudaMemcpyHostToDevice, c->st));
  const bool fp64 = precision == THR_FP64;
  const int epi = mode == 0 ? (norm2 ? 2 : 0) : mode;
  auto run = [&](auto* o, const auto* i, const auto* a, const auto* u) -> int {
    using S = std::remove_cv_t<std::remove_pointer_t<decltype(o)>>;
    if (epi == 0) return launch_dslash<S>(c->g, c->p.kernel, dag != 0, o, i, u, am, imass, c->p.am3, c->st);
    if (epi == 2)
      return launch_dslash_norm<S>(c->g, c->p.kernel, dag != 0, o, i, u, am, imass, c->p.am3, c->st, nullptr,
                                   c->partials);
    if (epi == 1)
      return launch_dslash_axpy<S>(c->g, c->p.kernel, dag != 0, o, i, u, am, imass, c->p.am3, c->st, nullptr, a,
                                   dcoef, c->partials);
    return launch_dslash_accum<S>(c->g, c->p.kernel, dag != 0, o, i, u, am, imass, c->p.am3, c->st, nullptr, a,
                                  dcoef, c->partials);
  };
  int rc;
  switch (precision) {
    case THR_FP64:
      rc = run((double2*)out, (const double2*)in, (const double2*)aux, (const double2*)c->u64);
      break;
    case THR_FP32_REF:
    case THR_MIXED_FP32:
      rc = run((float2*)out, (const float2*)in, (const float2*)aux, (const float2*)c->u32);
      break;
    case THR_MIXED_BF16:
      rc = run((__nv_bfloat162*)out, (const __nv_bfloat162*)in, (const __nv_bfloat162*)aux, (const float2*)c->u32);
      break;
    default: return THR_ERR_BADARG;
  }
  if (rc) return rc;
  if (epi != 0) {
    finish_sum(c->partials, (int)stencil_parts(c->g, c->p.kernel, fp64), dsum, c->st);
    THR_CUDA(cudaMemcpyAsync(c->hscal + kScalFusedSum, dsum, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    THR_TRY(c->sync());
    *norm2 = c->hscal[kScalFusedSum];
  }
  return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
}

int thr_sync(thr_ctx* c) {
  if (!c) return THR_ERR_BADARG;
  return c->sync();
}

int thr_profile(thr_ctx* c, int stride, int reset) {
  if (!c || stride < 0) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  if (reset) {
    cudaStreamSynchronize(c->st);
    c->prof_kind.clear();
    c->prof_bytes.clear();
    c->prof_tag.clear();
    for (long long& n : c->prof_seen) n = 0;
    for (double& n : c->prof_work) n = 0.0;
  }
  c->prof_on = stride != 0;
  if (stride > 0) c->prof_stride = stride;
  return THR_OK;
}

int thr_profile_read(thr_ctx* c, int kind, int* sampled, double* ms, double* bytes, double* launches) {
  if (!c || kind < 0 || kind >= thr_ctx::P_COUNT) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  THR_CUDA(cudaStreamSynchronize(c->st));
  int cnt = 0;
  double tot = 0.0, byt = 0.0;
  for (size_t i = 0; i < c->prof_kind.size(); i++) {
    if (c->prof_kind[i] != kind) continue;
    float e = 0.0f;
    THR_CUDA(cudaEventElapsedTime(&e, c->prof_ev[2 * i], c->prof_ev[2 * i + 1]));
    tot += e;
    byt += c->prof_bytes[i];
    cnt++;
  }
  if (sampled) *sampled = cnt;
  if (ms) *ms = tot;
  if (bytes) *bytes = byt;
  if (launches) *launches = c->prof_work[kind];
  return THR_OK;
}

int thr_get_stream(thr_ctx* c, void** s) {
  if (!c || !s) return THR_ERR_BADARG;
  *s = (void*)c->st;
  return THR_OK;
}

}  // extern "C"
