// qmr.cu -- qmrherm (qmrherm_module.F90:20-197), the multishift entry points
// and derivs, on device fields, plus their C ABI wrappers.
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ctx.h"
#include "derivs.h"
#include "ms.h"
#include "qmr.h"
#include "solver.h"

namespace thr {

namespace {
constexpr int kThreads = 256;
inline unsigned vec_grid(size_t n) {
  size_t b = (n + kThreads - 1) / kThreads;
  if (b > device_sms() * 16) b = device_sms() * 16;
  return (unsigned)(b ? b : 1);
}

struct Coefs {
  double a[kMaxShift + 1];
};

// x = anum(0)*Phi (:83) then x += anum(k)*x1(k) for k = 1..nq in order (:96-100)
__global__ void k_qmr_combine(double2* x, const double2* Phi, const double2* x1, size_t n, size_t stride, int nq,
                              Coefs c, int add_shifts) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double2 v = c.a[0] * Phi[i];
    if (add_shifts)
      for (int k = 0; k < nq; k++) v = v + c.a[k + 1] * x1[k * stride + i];
    x[i] = v;
  }
}
// a = Phi - sigma * x (the shifted part of the true residual)
__global__ void k_shift_part(double2* a, const double2* Phi, const double2* x, double sigma, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    a[i] = Phi[i] - sigma * x[i];
}
__global__ void k_f2d(double2* d, const float2* s, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    d[i] = make_double2((double)s[i].x, (double)s[i].y);
}
__global__ void k_d2f(float2* d, const double2* s, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    d[i] = make_float2((float)s[i].x, (float)s[i].y);
}
}  // namespace

// Multishift into x1 (FP64, nq fields of n).  sp: 0 FP64; 1 multishift_solver_sp
// (FP32 vectors throughout, the reference's single-precision solver); 2, 3 the
// mixed solver (FP64, then an FP32 / BF16-storage base iteration once the residual
// is small, FP64 shift fields; batched organisation only, else FP64)
int multishift_into(thr_ctx* c, const double2* Phi, double2* x1, int nq, const double* aden, const double* anum,
                    float res, float am, int imass, int maxcg, int sp, int* itercg, int* cg_returns) {
  const size_t n = c->n4();
  const bool batched = c->ms_algo == 1;
  c->mixed_switched_at = 0;
  if ((sp == 2 || sp == 3) && batched) {
    void *sf, *ring, *w32;
    THR_TRY(c->buffer(thr_ctx::B_SF64, (size_t)nq * n * sizeof(double2), &sf));
    THR_TRY(c->ensure_w64(8));
    THR_TRY(c->buffer(thr_ctx::B_RING, (size_t)(2 * kBatch) * n * sizeof(double2), &ring));
    THR_TRY(c->buffer(thr_ctx::B_WORK32, 5 * n * sizeof(float2), &w32));
    if (sp == 2)
      return multishift_mixed_dev<float2>(c, Phi, x1, (double2*)sf, (double2*)ring, c->w64[5], c->w64[6], c->w64[7],
                                          (float2*)w32, nq, aden, anum, res, am, imass, maxcg, c->mixed_switch[0],
                                          itercg, cg_returns, &c->mixed_switched_at);
    return multishift_mixed_dev<__nv_bfloat162>(c, Phi, x1, (double2*)sf, (double2*)ring, c->w64[5], c->w64[6],
                                                c->w64[7], (__nv_bfloat162*)w32, nq, aden, anum, res, am, imass,
                                                maxcg, c->mixed_switch[1], itercg, cg_returns, &c->mixed_switched_at);
  }
  if (sp != 1) {
    void *sf, *ring;
    THR_TRY(c->buffer(thr_ctx::B_SF64, (size_t)nq * n * sizeof(double2), &sf));
    THR_TRY(c->ensure_w64(8));
    if (batched) {
      THR_TRY(c->buffer(thr_ctx::B_RING, (size_t)(2 * kBatch) * n * sizeof(double2), &ring));
      return multishift_batched_dev<double2>(c, Phi, x1, (double2*)sf, (double2*)ring, c->w64[5], c->w64[6],
                                             c->w64[7], nq, aden, anum, res, am, imass, maxcg, itercg, cg_returns);
    }
    return multishift_dev<double2>(c, nullptr, Phi, x1, (double2*)sf, c->w64[4], c->w64[5], c->w64[6], c->w64[7], nq,
                                   aden, anum, res, am, imass, maxcg, itercg, cg_returns);
  }
  void *out32, *sf32, *w32;
  THR_TRY(c->buffer(thr_ctx::B_OUT32, (size_t)nq * n * sizeof(float2), &out32));
  THR_TRY(c->buffer(thr_ctx::B_SF32, (size_t)nq * n * sizeof(float2), &sf32));
  THR_TRY(c->buffer(thr_ctx::B_WORK32, 5 * n * sizeof(float2), &w32));
  float2* w = (float2*)w32;
  k_d2f<<<vec_grid(n), kThreads, 0, c->st>>>(w + 4 * n, Phi, n);  // input = cmplx(inputdp)
  int rc;
  if (batched) {
    void* ring;
    THR_TRY(c->buffer(thr_ctx::B_RING, (size_t)(2 * kBatch) * n * sizeof(double2), &ring));
    rc = multishift_batched_dev<float2>(c, w + 4 * n, (float2*)out32, (float2*)sf32, (float2*)ring, w, w + n,
                                        w + 2 * n, nq, aden, anum, res, am, imass, maxcg, itercg, cg_returns);
  } else {
    rc = multishift_dev<float2>(c, nullptr, w + 4 * n, (float2*)out32, (float2*)sf32, w, w + n, w + 2 * n, w + 3 * n,
                                nq, aden, anum, res, am, imass, maxcg, itercg, cg_returns);
  }
  k_f2d<<<vec_grid((size_t)nq * n), kThreads, 0, c->st>>>(x1, (const float2*)out32, (size_t)nq * n);
  return rc;
}

// r2[k] = |Phi - (M^dagger M + aden[k]) x_k|^2 in FP64 for the nq fields x_k
int shift_residuals(thr_ctx* c, const double2* Phi, const double2* x1, int nq, const double* aden, float am, int imass,
                    double* r2) {
  const size_t n = c->n4();
  THR_TRY(c->ensure_w64(10));
  double2 *t = c->w64[8], *a = c->w64[9];
  double* dcoef = c->dscal + kScalFusedCoef;
  double* dsum = c->dscal + kScalFusedSum;
  const double minus_one = -1.0;
  THR_CUDA(cudaMemcpyAsync(dcoef, &minus_one, sizeof(double), cudaMemcpyHostToDevice, c->st));
  const int np = (int)stencil_parts(c->g, c->p.kernel, true);
  for (int k = 0; k < nq; k++) {
    const double2* xk = x1 + (size_t)k * n;
    k_shift_part<<<vec_grid(n), kThreads, 0, c->st>>>(a, Phi, xk, aden[k], n);
    THR_TRY(launch_dslash<double2>(c->g, c->p.kernel, false, t, xk, c->u64, am, imass, c->p.am3, c->st));
    // a = a - M^dagger t, with |a|^2 per block
    THR_TRY(launch_dslash_axpy<double2>(c->g, c->p.kernel, true, a, t, c->u64, am, imass, c->p.am3, c->st, nullptr, a,
                                        dcoef, c->partials));
    finish_sum(c->partials, np, dsum, c->st);
    THR_CUDA(cudaMemcpyAsync(c->hscal + kScalFusedSum, dsum, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    THR_TRY(c->sync());
    r2[k] = c->hscal[kScalFusedSum];
  }
  return THR_OK;
}

int qmrherm_dev(thr_ctx* c, const double2* Phi, double2* x, float res, int* itercg, float am, int imass,
                const double* anum, const double* aden, int nq, int iflag, int use_sp, int* cg_returns, double* dS,
                int max_iters) {
  if (nq > c->p.ndiag || nq < 1 || nq > kMaxShift) return THR_ERR_BADSHAPE;  // :66-73
  if (c->g.ls % 4 != 0) return THR_ERR_BADSHAPE;                             // :75-81
  if (iflag < 0 || iflag > 3) return THR_ERR_BADARG;
  const size_t n = c->n4();
  // the reference's SP solver is Shamir-only (:53-63); the mixed modes take either kernel
  const int sp = use_sp == 1 ? (c->p.kernel == 0 ? 1 : 0) : (use_sp == 2 || use_sp == 3) ? use_sp : 0;
  void *x1v, *phi0v;
  THR_TRY(c->buffer(thr_ctx::B_X1, (size_t)nq * n * sizeof(double2), &x1v));
  double2* x1 = (double2*)x1v;
  std::vector<int> cgr(nq, 0);
  int rc = multishift_into(c, Phi, x1, nq, aden, anum + 1, res, am, imass, max_iters, sp, itercg, cgr.data());
  if (rc != THR_OK) return rc;
  if (cg_returns) memcpy(cg_returns, cgr.data(), nq * sizeof(int));
  Coefs cf;
  for (int k = 0; k <= nq; k++) cf.a[k] = anum[k];
  k_qmr_combine<<<vec_grid(n), kThreads, 0, c->st>>>(x, Phi, x1, n, n, nq, cf, iflag < 2);
  if (iflag == 1) {  // :111-113, Phi0 persists in the context like the module variable
    THR_TRY(c->buffer(thr_ctx::B_PHI0, (size_t)c->p.ndiag * n * sizeof(double2), &phi0v));
    THR_CUDA(cudaMemcpyAsync(phi0v, x1, (size_t)nq * n * sizeof(double2), cudaMemcpyDeviceToDevice, c->st));
    c->phi0_valid = true;
  }
  if (iflag >= 2) {
    if (!dS) return THR_ERR_BADARG;
    THR_TRY(c->ensure_w64(4));
    double2* x2 = c->w64[2];
    double2* Rb = c->w64[3];
    double2* phi0 = nullptr;
    if (iflag == 3) {
      THR_TRY(c->buffer(thr_ctx::B_PHI0, (size_t)c->p.ndiag * n * sizeof(double2), &phi0v));
      phi0 = (double2*)phi0v;
    }
    for (int k = 0; k < nq; k++) {
      const double2* xk = x1 + (size_t)k * n;
      THR_TRY(launch_dslash<double2>(c->g, c->p.kernel, false, x2, xk, c->u64, am, imass, c->p.am3, c->st));
      if (iflag == 2) {
        THR_TRY(launch_derivs(c, dS, xk, x2, anum[k + 1], 0, am, imass));  // :150-155
      } else {
        const double coeff = -anum[k + 1];
        const double2* pk = phi0 + (size_t)k * n;
        THR_TRY(launch_derivs(c, dS, pk, x2, coeff, 0, am, imass));  // :158-163
        THR_TRY(launch_dslash<double2>(c->g, c->p.kernel, false, Rb, pk, c->u64, am, imass, c->p.am3, c->st));
        THR_TRY(launch_derivs(c, dS, Rb, xk, coeff, 1, am, imass));  // :166-181
      }
    }
  }
  return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
}

}  // namespace thr

using namespace thr;

namespace {
int upload_d3(thr_ctx* c, double* dev, const double* host) {
  size_t n3 = (size_t)c->g.v3 * 3;
  THR_CUDA(cudaMemcpyAsync(c->stage, host, n3 * sizeof(double), cudaMemcpyHostToDevice, c->st));
  from_fortran_d3(c->g, dev, (const double*)c->stage, c->st);
  return THR_OK;
}
int download_d3(thr_ctx* c, double* host, const double* dev) {
  size_t n3 = (size_t)c->g.v3 * 3;
  to_fortran_d3(c->g, (double*)c->stage, dev, c->st);
  THR_CUDA(cudaMemcpyAsync(host, c->stage, n3 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  return THR_OK;
}
int dsdpi_dev(thr_ctx* c, double** out) {
  void* p;
  THR_TRY(c->buffer(thr_ctx::B_DSDPI, (size_t)c->g.v3 * 3 * sizeof(double), &p));
  *out = (double*)p;
  return THR_OK;
}
}  // namespace

extern "C" {

int thr_derivs(thr_ctx* c, const double* R, const double* X2, double anum, int iflag, float am, int imass,
               double* dSdpi) {
  if (!c || !R || !X2) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  THR_TRY(c->ensure_w64(2));
  double* dS;
  THR_TRY(dsdpi_dev(c, &dS));
  THR_TRY(c->upload_spinor(c->w64[0], R));
  THR_TRY(c->upload_spinor(c->w64[1], X2));
  if (dSdpi) THR_TRY(upload_d3(c, dS, dSdpi));
  THR_TRY(launch_derivs(c, dS, c->w64[0], c->w64[1], anum, iflag, am, imass));
  if (dSdpi) THR_TRY(download_d3(c, dSdpi, dS));
  return c->sync();
}

int thr_derivs_dev(thr_ctx* c, const void* R, const void* X2, double anum, int iflag, float am, int imass) {
  if (!c || !R || !X2) return THR_ERR_BADARG;
  if (!c->links_ok) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  double* dS;
  THR_TRY(dsdpi_dev(c, &dS));
  return launch_derivs(c, dS, (const double2*)R, (const double2*)X2, anum, iflag, am, imass);
}

static int ms_abi(thr_ctx* c, const double* u, float am, int imass, int ndiagq, const double* aden, const double* anum,
                  double* output, const double* input, float res, int maxcg, int* cg_return, int* cg_returns,
                  int sp) {
  if (!c || !aden || !anum || !output || !input || !cg_return) return THR_ERR_BADARG;
  if (ndiagq < 1 || ndiagq > c->p.ndiag || ndiagq > kMaxShift) return THR_ERR_BADSHAPE;
  cudaSetDevice(c->dev);
  THR_TRY(c->ensure_w64(8));
  THR_TRY(c->use_links(u));
  THR_TRY(c->upload_spinor(c->w64[0], input));
  void* x1;
  const size_t n = c->n4();
  THR_TRY(c->buffer(thr_ctx::B_X1, (size_t)ndiagq * n * sizeof(double2), &x1));
  int rc = multishift_into(c, c->w64[0], (double2*)x1, ndiagq, aden, anum, res, am, imass, maxcg, sp, cg_return,
                           cg_returns);
  if (rc) return rc;
  // output(:,:,:,:,:,1:ndiag) = 0 then the ndiagq solutions (multishift_module.F90:82)
  memset(output, 0, (size_t)c->p.ndiag * n * sizeof(double2));
  for (int k = 0; k < ndiagq; k++) {
    to_fortran_noh(c->g, c->stage, (const double2*)x1 + (size_t)k * n, c->st);
    THR_CUDA(cudaMemcpyAsync(output + 2 * (size_t)k * n, c->stage, n * sizeof(double2), cudaMemcpyDeviceToHost, c->st));
  }
  return c->sync();
}

int thr_multishift_solver(thr_ctx* c, const double* u, float am, int imass, int ndiagq, const double* aden,
                          const double* anum, double* output, const double* input, float res, int maxcg,
                          int* cg_return, int* cg_returns) {
  return ms_abi(c, u, am, imass, ndiagq, aden, anum, output, input, res, maxcg, cg_return, cg_returns, 0);
}
int thr_multishift_solver_sp(thr_ctx* c, const double* u, float am, int imass, int ndiagq, const double* aden,
                             const double* anum, double* output, const double* input, float res, int maxcg,
                             int* cg_return, int* cg_returns) {
  return ms_abi(c, u, am, imass, ndiagq, aden, anum, output, input, res, maxcg, cg_return, cg_returns, 1);
}

int thr_qmrherm(thr_ctx* c, const double* Phi, double* x, float res, int* itercg, float am, int imass,
                const double* anum, const double* aden, int ndiagq, int iflag, int use_sp, int* cg_returns,
                double* dSdpi, double* Phi0, int max_qmr_iters) {
  if (!c || !Phi || !x || !itercg || !anum || !aden) return THR_ERR_BADARG;
  if (imass != 1 && imass != 3 && imass != 5) return THR_ERR_BADARG;
  if (ndiagq > c->p.ndiag || ndiagq < 1 || ndiagq > kMaxShift) return THR_ERR_BADSHAPE;
  if (c->g.ls % 4 != 0) return THR_ERR_BADSHAPE;
  cudaSetDevice(c->dev);
  THR_TRY(c->ensure_w64(8));
  THR_TRY(c->use_links(nullptr));
  const size_t n = c->n4();
  double2* dPhi = c->w64[0];
  double2* dx = c->w64[1];
  THR_TRY(c->upload_spinor(dPhi, Phi));
  double* dS = nullptr;
  if (iflag >= 2) {
    THR_TRY(dsdpi_dev(c, &dS));
    if (dSdpi) THR_TRY(upload_d3(c, dS, dSdpi));
    if (iflag == 3 && Phi0) {  // Phi0(…, 1:ndiagq) from the caller
      void* p0;
      THR_TRY(c->buffer(thr_ctx::B_PHI0, (size_t)c->p.ndiag * n * sizeof(double2), &p0));
      for (int k = 0; k < ndiagq; k++)
        THR_TRY(c->upload_spinor((double2*)p0 + (size_t)k * n, Phi0 + 2 * (size_t)k * c->nf5()));
    } else if (iflag == 3 && !c->phi0_valid) {
      return THR_ERR_BADARG;
    }
  }
  if (max_qmr_iters <= 0) max_qmr_iters = 50000;  // params.F90:56
  int rc = qmrherm_dev(c, dPhi, dx, res, itercg, am, imass, anum, aden, ndiagq, iflag, use_sp, cg_returns, dS,
                       max_qmr_iters);
  if (rc) return rc;
  THR_TRY(c->download_spinor(x, dx));
  if (iflag == 1 && Phi0) {
    void* p0;
    THR_TRY(c->buffer(thr_ctx::B_PHI0, (size_t)c->p.ndiag * n * sizeof(double2), &p0));
    for (int k = 0; k < ndiagq; k++)
      THR_TRY(c->download_spinor(Phi0 + 2 * (size_t)k * c->nf5(), (const double2*)p0 + (size_t)k * n));
  }
  if (iflag >= 2 && dSdpi) THR_TRY(download_d3(c, dSdpi, dS));
  return c->sync();
}

int thr_set_mixed(thr_ctx* c, double switch_fp32, double switch_bf16) {
  if (!c || !(switch_fp32 >= 0.0) || !(switch_bf16 >= 0.0)) return THR_ERR_BADARG;
  c->mixed_switch[0] = switch_fp32;
  c->mixed_switch[1] = switch_bf16;
  return THR_OK;
}

int thr_mixed_switched_at(thr_ctx* c, int* iteration) {
  if (!c || !iteration) return THR_ERR_BADARG;
  *iteration = c->mixed_switched_at;
  return THR_OK;
}

int thr_set_solver(thr_ctx* c, int multishift_algo) {
  if (!c || multishift_algo < 0 || multishift_algo > 2) return THR_ERR_BADARG;
  c->ms_algo = multishift_algo == 0 ? 0 : 1;
  const char* e = std::getenv("THR_GRAPHS");
  c->use_graphs = multishift_algo == 1 && !(e && e[0] == '0');
  return THR_OK;
}

int thr_shift_residuals_dev(thr_ctx* c, const void* Phi, const void* x, int nq, const double* aden, float am,
                            int imass, double* r2) {
  if (!c || !Phi || !aden || !r2 || nq < 1) return THR_ERR_BADARG;
  if (imass != 1 && imass != 3 && imass != 5) return THR_ERR_BADARG;
  if (!c->links_ok) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  const size_t n = c->n4();
  const double2* x1 = (const double2*)x;
  if (!x1) {  // the context's last multishift solutions (qmrherm's x1)
    if (c->buf_bytes[thr_ctx::B_X1] < (size_t)nq * n * sizeof(double2)) return THR_ERR_BADARG;
    x1 = (const double2*)c->bufs[thr_ctx::B_X1];
  }
  return shift_residuals(c, (const double2*)Phi, x1, nq, aden, am, imass, r2);
}

int thr_qmrherm_dev(thr_ctx* c, const void* Phi, void* x, float res, int* itercg, float am, int imass,
                    const double* anum, const double* aden, int ndiagq, int iflag, int use_sp, int* cg_returns) {
  if (!c || !Phi || !x || !itercg || !anum || !aden) return THR_ERR_BADARG;
  if (imass != 1 && imass != 3 && imass != 5) return THR_ERR_BADARG;
  if (iflag >= 2) {
    if (iflag == 3 && !c->phi0_valid) return THR_ERR_BADARG;
  }
  cudaSetDevice(c->dev);
  if (!c->links_ok) return THR_ERR_BADARG;
  double* dS = nullptr;
  if (iflag >= 2) THR_TRY(dsdpi_dev(c, &dS));
  return qmrherm_dev(c, (const double2*)Phi, (double2*)x, res, itercg, am, imass, anum, aden, ndiagq, iflag, use_sp,
                     cg_returns, dS, c->max_qmr_iters);
}

}  // extern "C"
