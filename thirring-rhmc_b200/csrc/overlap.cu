// overlap.cu -- the overlap (Zolotarev domain-wall) operator of
// measure_OWilson.F90: the slice coefficients of prepZolo (:169-188), odslash
// and odslashd (:14-167, stencil in dslash.cu) and congradO (:190-268).
//
// The coefficients c[s] = 1 / root[s] come from the Zolotarev optimal rational
// approximation of sign(x) on [lmin, lmax] with N = Ls roots (Chiu's formula for
// the roots with Kennedy's lambda, ZOLO/zolomodule.f:26-65, :196-251).  The
// reference evaluates the elliptic functions it needs by published
// approximations, and the same ones are used here so that the coefficients
// agree with its:
//   K(k)        Hastings' polynomial approximation, Abramowitz & Stegun 17.3.34
//               (ZOLO/ellipticmodule.f:114-197), accurate to ~2e-8;
//   sn(u | k)   the arithmetic-geometric mean with descending Landen
//               transformations, A&S 16.4, stopped when c < 1e-7 (:19-112);
//   arcsn(x|k)  the integral of 1/sqrt((1-t^2)(1-k^2 t^2)) from 0 to x by
//               3-point Gauss-Legendre quadrature on 10000 panels (:409-438).
#include <cmath>
#include <vector>

#include <algorithm>

#include "ctx.h"
#include "overlap.h"
#include "rng.h"
#include "thr_reduce.cuh"

namespace thr {

namespace {

// ---------------------------------------------------------------- elliptic functions
double ell_k(double k) {
  if (k == 1.0) return 1.0e300;
  const double m1 = 1.0 - k * k;  // complementary parameter
  static const double a[5] = {1.38629436112, 0.09666344259, 0.03590092383, 0.03742563713, 0.01451196212};
  static const double b[5] = {0.5, 0.12498593597, 0.06880248576, 0.03328355346, 0.00441787012};
  double pa = a[4], pb = b[4];
  for (int i = 3; i >= 0; i--) {
    pa = pa * m1 + a[i];
    pb = pb * m1 + b[i];
  }
  return pa - pb * std::log(m1);
}

struct SnDn {
  double sn, dn;
};
SnDn ell_sn(double u, double k) {
  double ratio[41];
  double am = 1.0, bm = std::sqrt(1.0 - k * k), a = 1.0;
  int steps = 0;
  while (steps < 40) {
    steps++;
    a = 0.5 * (am + bm);
    const double g = std::sqrt(am * bm), c = 0.5 * (am - bm);
    ratio[steps] = c / a;
    if (c < 1.0e-7) break;
    am = a;
    bm = g;
  }
  double phi = std::ldexp(a * u, steps);
  for (int j = steps; j >= 1; j--) {
    const double t = ratio[j] * std::sin(phi);
    phi = 0.5 * (phi + std::atan(t / std::sqrt(std::fabs(1.0 - t * t))));
  }
  const double sn = std::sin(phi);
  return {sn, std::sqrt(1.0 - k * k * sn * sn)};
}

double ell_arcsn(double x, double k, int panels) {
  auto f = [k](double t) { return std::pow((1.0 + t) * (1.0 - t), -0.5) * std::pow((1.0 + k * t) * (1.0 - k * t), -0.5); };
  const double h = x / panels, off = std::sqrt(3.0 / 5.0) * h / 2.0;
  double t = h / 2.0, sum = 0.0;
  for (int i = 0; i < panels; i++) {
    sum += (5.0 / 9.0 * f(t - off) + 8.0 / 9.0 * f(t) + 5.0 / 9.0 * f(t + off)) * h / 2.0;
    t += h;
  }
  return sum;
}

// R(x) of zolomodule.f:114-123: prod over the N/2 pairs of (1 - x/cnum) / (1 - x/cdenom)
double zolo_pairs(double x, const std::vector<double>& cnum, const std::vector<double>& cden) {
  double v = 1.0;
  for (size_t l = 0; l < cnum.size(); l++) v = v * (1.0 - x / cnum[l]) / (1.0 - x / cden[l]);
  return v;
}

}  // namespace

int zolo_coefficients(int n, double lmin, double lmax, double* out) {
  if (n < 1 || !(lmin > 0.0) || !(lmax > lmin) || !out) return THR_ERR_BADARG;
  // setZolo (zolomodule.f:26-65)
  const double beta = lmax / lmin, k = 1.0 / beta;
  const double kd = std::sqrt(1.0 - k) * std::sqrt(1.0 + k);
  const double bigK = ell_k(k), bigKd = ell_k(kd);
  std::vector<double> cnum(n / 2), cden(n / 2);
  auto pole = [](double s) { return -s / (1.0 - s) * s / (1.0 + s); };
  for (int l = 0; l < n / 2; l++) {  // setInnerCoeffs (:67-94)
    cnum[l] = pole(ell_sn((2 * l + 2) * bigKd / n, kd).sn);
    cden[l] = pole(ell_sn((2 * l + 1) * bigKd / n, kd).sn);
  }
  const double M = zolo_pairs(1.0, cnum, cden);  // calcM
  const SnDn e = ell_sn(bigK, k), dd = ell_sn(bigKd / n, kd);
  const double C = e.sn * dd.dn / (1.0 - e.dn * e.dn * dd.sn * dd.sn);  // calcC (:135-154)
  const double lambda = M / (C * zolo_pairs(C * C, cnum, cden));      // calcLambda
  // getRoots (:196-251)
  const double l1 = 1.0 + lambda;
  const double arg = std::sqrt((1.0 + 3.0 * lambda) / (l1 * l1 * l1));
  const double c1 = M * ell_arcsn(arg, std::sqrt(l1 * (1.0 - lambda)), 10000);
  const double c2 = 2.0 * bigKd / n;
  for (int s = 0; s < n; s++) {
    const double v = (s % 2 == 0 ? c1 : -c1) + ((s + 1) / 2) * c2;
    const double sn = ell_sn(v, kd).sn;
    const double root = 1.0 / (std::sqrt(1.0 - kd * kd * sn * sn) / lmin);
    out[s] = 1.0 / root;  // coeffs = 1d0/zolo%roots (measure_OWilson.F90:182)
  }
  return THR_OK;
}

// the context's coefficients on the device (prepZolo's defaults unless set)
int zolo_device(thr_ctx* c, const double** zc) {
  if (c->zolo.empty()) {
    std::vector<double> h((size_t)c->g.ls);
    THR_TRY(zolo_coefficients(c->g.ls, 0.1, 5.0, h.data()));  // measure_OWilson.F90:179-180
    c->zolo = h;
    c->zolo_dirty = true;
  }
  if (!c->zolo_dev) {
    if (cudaMalloc(&c->zolo_dev, (size_t)c->g.ls * sizeof(double)) != cudaSuccess) return THR_ERR_NOMEM;
    c->zolo_dirty = true;
  }
  if (c->zolo_dirty) {
    THR_CUDA(cudaMemcpyAsync(c->zolo_dev, c->zolo.data(), (size_t)c->g.ls * sizeof(double), cudaMemcpyHostToDevice,
                             c->st));
    c->zolo_dirty = false;
  }
  *zc = c->zolo_dev;
  return THR_OK;
}

// ---------------------------------------------------------------- congradO
namespace {
constexpr int kThreads = 256;
constexpr int kChunk = 4;  // iterations between host checks
constexpr int kPartB = 8192;  // offset of the second set of partials

struct CgoState {
  double resid, alpha, alphan, alphad, betacg;
  int itercg, iters, done, niterc, status;
};

inline unsigned vgrid(size_t n) {
  size_t b = (n + kThreads - 1) / kThreads;
  if (b > device_sms() * 8) b = device_sms() * 8;
  return (unsigned)(b ? b : 1);
}

// r = Phi - x2, p = r, partials of |r|^2
__global__ void k_cgo_start(double2* r, double2* p, const double2* phi, const double2* x2, size_t n, double* partials) {
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double2 v = phi[i] - x2[i];
    r[i] = v;
    p[i] = v;
    acc += v.x * v.x + v.y * v.y;
  }
  block_write_partial(acc, partials);
}
// betacgn of the start; converged before the loop: iterations = 0
__global__ void k_cgo_init(CgoState* cs, const double* partials, int np) {
  const double b = block_sum_partials(partials, np);
  if (threadIdx.x == 0) {
    cs->alphan = b;  // the first iteration's alphan = |r|^2 (:232)
    if (b < cs->resid) {
      cs->done = 1;
      cs->iters = 0;
    }
  }
}
// alphad = Re<p, x2> (:234-235), alpha = alphan / alphad
__global__ void k_cgo_alpha(CgoState* cs, const double* partials, int np) {
  if (cs->done) return;
  const double d = block_sum_partials(partials, np);
  if (threadIdx.x == 0) {
    cs->itercg += 1;
    cs->alphad = d;
    cs->alpha = cs->alphan / d;
  }
}
// x = x + alpha p, r = r - alpha x2 (:238-239), partials of |r|^2
__global__ void k_cgo_xr(const CgoState* cs, double2* x, double2* r, const double2* p, const double2* x2, size_t n,
                         double* partials) {
  if (cs->done) return;
  const double a = cs->alpha;
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    x[i] = x[i] + a * p[i];
    const double2 v = r[i] - a * x2[i];
    r[i] = v;
    acc += v.x * v.x + v.y * v.y;
  }
  block_write_partial(acc, partials);
}
// betacgn, the stopping test (:247), betacg = betacgn / alphan (:248)
__global__ void k_cgo_beta(CgoState* cs, const double* partials, int np) {
  if (cs->done) return;
  const double b = block_sum_partials(partials, np);
  if (threadIdx.x == 0) {
    if (b < cs->resid) {
      cs->done = 1;
      cs->iters = cs->itercg;
    } else if (cs->itercg >= cs->niterc) {
      cs->done = 1;
      cs->iters = cs->niterc + 1;  // the loop ran out (:250)
      cs->status = THR_ERR_MAXITER;
    } else {
      cs->betacg = b / cs->alphan;
      cs->alphan = b;  // the next iteration's |r|^2
    }
  }
}
// p = r + betacg p (:249)
__global__ void k_cgo_p(const CgoState* cs, double2* p, const double2* r, size_t n) {
  if (cs->done) return;
  const double b = cs->betacg;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    p[i] = r[i] + b * p[i];
}
}  // namespace

// congradO on device fields: X = solution (initial guess Phi, :216-217)
int congrad_o_dev(thr_ctx* c, const double2* phi, double2* X, float res, float am, int imass, int niterc, int* itercg,
                  int* iterations) {
  const double* zc = nullptr;
  THR_TRY(zolo_device(c, &zc));
  THR_TRY(c->ensure_w64(8));
  double2 *x1 = c->w64[4], *x2 = c->w64[5], *p = c->w64[6], *r = c->w64[7];
  const size_t n = c->n4();
  const unsigned gb = vgrid(n);
  CgoState* cs = reinterpret_cast<CgoState*>(c->dscal);
  CgoState h{};
  const int ivol = 4 * c->g.lx * c->g.ly * c->g.lt * c->g.ls;
  const float resid = ((float)ivol * res) * res;  // :214, default real
  h.resid = (double)resid;
  h.niterc = niterc;
  THR_CUDA(cudaMemcpyAsync(cs, &h, sizeof(CgoState), cudaMemcpyHostToDevice, c->st));
  THR_CUDA(cudaMemcpyAsync(X, phi, n * sizeof(double2), cudaMemcpyDeviceToDevice, c->st));  // x = r = Phi
  THR_TRY(launch_odslash(c->g, false, x1, X, c->u64, am, imass, c->p.am3, zc, c->st));
  THR_TRY(launch_odslash(c->g, true, x2, x1, c->u64, am, imass, c->p.am3, zc, c->st));
  k_cgo_start<<<gb, kThreads, 0, c->st>>>(r, p, phi, x2, n, c->partials);
  k_cgo_init<<<1, 1024, 0, c->st>>>(cs, c->partials, gb);
  for (;;) {
    for (int k = 0; k < kChunk; k++) {
      THR_TRY(launch_odslash(c->g, false, x1, p, c->u64, am, imass, c->p.am3, zc, c->st, &cs->done));
      THR_TRY(launch_odslash(c->g, true, x2, x1, c->u64, am, imass, c->p.am3, zc, c->st, &cs->done));
      const int nb = redot_partials<double2>(p, x2, n, c->partials + kPartB, c->st);
      k_cgo_alpha<<<1, 1024, 0, c->st>>>(cs, c->partials + kPartB, nb);
      k_cgo_xr<<<gb, kThreads, 0, c->st>>>(cs, X, r, p, x2, n, c->partials);
      k_cgo_beta<<<1, 1024, 0, c->st>>>(cs, c->partials, gb);
      k_cgo_p<<<gb, kThreads, 0, c->st>>>(cs, p, r, n);
    }
    THR_CUDA(cudaMemcpyAsync(&h, cs, sizeof(CgoState), cudaMemcpyDeviceToHost, c->st));
    THR_CUDA(cudaStreamSynchronize(c->st));
    if (h.done) break;
  }
  if (itercg) *itercg = h.itercg;
  if (iterations) *iterations = h.iters;
  return h.status ? h.status : THR_OK;
}

// ---------------------------------------------------------------- overlap measurement
// measure_wilsonKDDW (measure_OWilson.F90:646-673), the MEASURE_OWILSON branch of
// measure (measure_module.F90:158-160).  Per noise, evalSingleCondNoise_KDDW4
// (:704-757) draws gauss0 four times; the draw idx becomes eta on spin idx of the
// slice s = 1 of a 5D field (IKDDW4, :462-478) and
//   IKDDW = PermM^dag . IDDW(bmass) . odslash(mass 1, imass 1) . PermM   (:369-393)
//   IDDW(m) R = congradO(odslashd(m) R) at respbp                       (:270-289)
// is applied; the trace of conj(eta) (result - eta) over spin idx of the slice,
// divided by 1 - bmass (imass 1) or (-bmass, +-1) (imass 3), summed over idx and
// divided by kvol is the noise's psibarpsi.
namespace {
constexpr int kOwThreads = 256;

// R5 = 0 except slice 0, spin d: cmplx(ps(:,:,:,1), ps(:,:,:,2)) (:722-724)
__global__ void k_ow_source(double2* R5, const float* __restrict__ ps, Geom g, int d) {
  const int site = blockIdx.x * blockDim.x + threadIdx.x;
  if (site >= g.v3) return;
  R5[sidx(g, 0, site, d)] = make_double2((double)ps[site], (double)ps[g.v3 + site]);
}
// PermM (:546-576): out(s) = P- in(s) + P+ in(s+1) (s+1 past the last slice -> the
// first); dag: P+ in(s-1) (before the first -> the last).  P+ = spins 0,1.
__global__ void k_permm(double2* __restrict__ out, const double2* __restrict__ in, Geom g, int dag) {
  const size_t n = (size_t)g.ls * g.v3;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int s = (int)(e % g.ls);
    const int site = (int)(e / g.ls);
    const int sp = dag ? (s == 0 ? g.ls - 1 : s - 1) : (s == g.ls - 1 ? 0 : s + 1);
#pragma unroll
    for (int d = 0; d < 4; d++) out[sidx(g, s, site, d)] = in[sidx(g, d < 2 ? sp : s, site, d)];
  }
}
// partials per block of conj(eta) (DR(slice 0, spin d) - eta) (:725-747)
__global__ void __launch_bounds__(kOwThreads) k_ow_contract(const double2* __restrict__ DR, const float* __restrict__ ps,
                                                            Geom g, int d, double2* __restrict__ partials) {
  const int site = blockIdx.x * blockDim.x + threadIdx.x;
  double2 acc = make_double2(0.0, 0.0);
  if (site < g.v3) {
    const double2 eta = make_double2((double)ps[site], (double)ps[g.v3 + site]);
    acc = cjmul(eta, DR[sidx(g, 0, site, d)] - eta);
  }
  __shared__ double2 sh[kOwThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    acc.x += __shfl_down_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_down_sync(0xffffffffu, acc.y, o);
  }
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double2 v = sh[0];
    for (int w = 1; w < kOwThreads / 32; w++) v = v + sh[w];
    partials[blockIdx.x] = v;
  }
}
}  // namespace

int measure_ow(thr_ctx* c, float respbp, float bmass, int imass, int knoise, float* psibarpsi, float* susclsing,
               float* aviter, double* parts, int* itercg) {
  if (imass != 1 && imass != 3) return THR_ERR_BADARG;  // evalSingleCondNoise_KDDW4 :733-741
  const Geom& g = c->g;
  const double* zc = nullptr;
  THR_TRY(zolo_device(c, &zc));
  THR_TRY(c->ensure_w64(8));
  double2 *R5 = c->w64[0], *T = c->w64[1], *DR = c->w64[2], *IDR = c->w64[3];
  const size_t n4 = c->n4();
  const int nsolve = 4 * knoise;
  // every draw first, in the reference's order (the solves draw no random numbers)
  float* eta = nullptr;
  THR_CUDA(cudaMalloc(&eta, sizeof(float) * 2 * (size_t)g.v3 * nsolve));
  const unsigned nblk = (unsigned)((g.v3 + kOwThreads - 1) / kOwThreads);
  double2* part = nullptr;
  int rc = cudaMalloc(&part, sizeof(double2) * nblk) == cudaSuccess ? THR_OK : THR_ERR_NOMEM;
  for (int j = 0; !rc && j < nsolve; j++) rc = rng_gauss_dev(c, -1.0f, eta + (size_t)j * 2 * g.v3);
  const int niterc = g.ls * g.v3;  // params.F90:57
  std::vector<double2> hp(nblk);
  std::vector<double2> cpbp(knoise, make_double2(0.0, 0.0));
  std::vector<int> its(nsolve, 0);
  size_t pgrid = ((size_t)g.ls * g.v3 + kOwThreads - 1) / kOwThreads;
  if (pgrid > device_sms() * 8) pgrid = device_sms() * 8;
  for (int j = 0; !rc && j < nsolve; j++) {
    const int d = j % 4;
    const float* e = eta + (size_t)j * 2 * g.v3;
    if (cudaMemsetAsync(R5, 0, n4 * sizeof(double2), c->st) != cudaSuccess) { rc = THR_ERR_CUDA; break; }
    k_ow_source<<<nblk, kOwThreads, 0, c->st>>>(R5, e, g, d);
    k_permm<<<(unsigned)pgrid, kOwThreads, 0, c->st>>>(T, R5, g, 0);
    rc = launch_odslash(g, false, DR, T, c->u64, 1.0f, 1, c->p.am3, zc, c->st);  // DDW(1), mtype 1
    if (!rc) rc = launch_odslash(g, true, IDR, DR, c->u64, bmass, imass, c->p.am3, zc, c->st);
    if (rc) break;
    int it = 0, nx = 0;
    rc = congrad_o_dev(c, IDR, T, respbp, bmass, imass, niterc, &it, &nx);
    if (rc == THR_ERR_MAXITER) rc = THR_OK;  // congradO only prints a warning (:250)
    if (rc) break;
    its[j] = it;
    k_permm<<<(unsigned)pgrid, kOwThreads, 0, c->st>>>(DR, T, g, 1);
    k_ow_contract<<<nblk, kOwThreads, 0, c->st>>>(DR, e, g, d, part);
    if (cudaMemcpyAsync(hp.data(), part, sizeof(double2) * nblk, cudaMemcpyDeviceToHost, c->st) != cudaSuccess ||
        cudaStreamSynchronize(c->st) != cudaSuccess) {
      rc = THR_ERR_CUDA;
      break;
    }
    double2 tr = make_double2(0.0, 0.0);
    for (unsigned b = 0; b < nblk; b++) tr = tr + hp[b];
    // trcomp = sum / denom: denom = one - bmass in default real (imass 1), cmplx(-bmass, +-1) (imass 3)
    const double dr = imass == 1 ? (double)(1.0f - bmass) : -(double)bmass;
    const double di = imass == 1 ? 0.0 : (d < 2 ? 1.0 : -1.0);
    const double dd = dr * dr + di * di;
    cpbp[j / 4] = cpbp[j / 4] + make_double2((tr.x * dr + tr.y * di) / dd, (tr.y * dr - tr.x * di) / dd);
  }
  cudaFree(eta);
  cudaFree(part);
  if (rc) return rc;
  const double kvol = (double)g.v3;
  std::vector<double> vpbp(knoise);
  for (int n = 0; n < knoise; n++) {
    const double2 p = make_double2(cpbp[n].x / kvol, cpbp[n].y / kvol);
    vpbp[n] = p.x;
    if (parts) {
      parts[4 * n + 0] = p.x;
      parts[4 * n + 1] = p.y;
      parts[4 * n + 2] = 0.0;
      parts[4 * n + 3] = 0.0;
    }
  }
  double sum = 0.0;
  for (int n = 0; n < knoise; n++) sum += vpbp[n];
  float sus = 0.0f;  // output_OW (:683-687)
  for (int n = 0; n < knoise; n++) {
    double sv = 0.0;
    for (int m = n + 1; m < knoise; m++) sv += vpbp[n] * vpbp[m];
    sus = sus + (float)sv;
  }
  *psibarpsi = (float)(sum / knoise);  // pbp = sum(vpbp)/knoise (:669)
  *susclsing = (float)(2 * g.v3) * sus / (float)(knoise * (knoise - 1));
  *aviter = 0.0f;  // "not currently calculated" (:671)
  if (itercg) std::copy(its.begin(), its.end(), itercg);
  return THR_OK;
}

}  // namespace thr

using namespace thr;

extern "C" {

int thr_zolo_coeffs(int ls, double lmin, double lmax, double* coeffs) {
  return zolo_coefficients(ls, lmin, lmax, coeffs);
}

int thr_prep_zolo(thr_ctx* c, double lmin, double lmax) {
  if (!c) return THR_ERR_BADARG;
  std::vector<double> h((size_t)c->g.ls);
  THR_TRY(zolo_coefficients(c->g.ls, lmin, lmax, h.data()));
  c->zolo = h;
  c->zolo_dirty = true;
  return THR_OK;
}

int thr_zolo_get(thr_ctx* c, double* coeffs) {
  if (!c || !coeffs) return THR_ERR_BADARG;
  if (c->zolo.empty()) {
    std::vector<double> h((size_t)c->g.ls);
    THR_TRY(zolo_coefficients(c->g.ls, 0.1, 5.0, h.data()));
    c->zolo = h;
    c->zolo_dirty = true;
  }
  for (int s = 0; s < c->g.ls; s++) coeffs[s] = c->zolo[s];
  return THR_OK;
}

static int odslash_common(thr_ctx* c, double* Phi, const double* R, const double* u, float am, int imass, bool dag) {
  if (!c || !Phi || !R) return THR_ERR_BADARG;
  if (imass != 1 && imass != 3) return THR_ERR_BADARG;  // measure_OWilson.F90:66-83
  cudaSetDevice(c->dev);
  const double* zc = nullptr;
  THR_TRY(zolo_device(c, &zc));
  THR_TRY(c->ensure_w64(2));
  THR_TRY(c->use_links(u));
  THR_TRY(c->upload_spinor(c->w64[0], R));
  THR_TRY(launch_odslash(c->g, dag, c->w64[1], c->w64[0], c->u64, am, imass, c->p.am3, zc, c->st));
  THR_TRY(c->download_spinor(Phi, c->w64[1]));
  return c->sync();
}

int thr_odslash(thr_ctx* c, double* Phi, const double* R, const double* u, float am, int imass) {
  return odslash_common(c, Phi, R, u, am, imass, false);
}
int thr_odslashd(thr_ctx* c, double* Phi, const double* R, const double* u, float am, int imass) {
  return odslash_common(c, Phi, R, u, am, imass, true);
}

int thr_odslash_dev(thr_ctx* c, void* out, const void* in, float am, int imass, int dag) {
  if (!c || !out || !in) return THR_ERR_BADARG;
  if (imass != 1 && imass != 3) return THR_ERR_BADARG;
  if (!c->links_ok) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  const double* zc = nullptr;
  THR_TRY(zolo_device(c, &zc));
  return launch_odslash(c->g, dag != 0, (double2*)out, (const double2*)in, c->u64, am, imass, c->p.am3, zc, c->st);
}

int thr_congrad_o(thr_ctx* c, const double* Phi, double* X, float res, int* itercg, float am, int imass,
                  int* iterations) {
  if (!c || !Phi || !X) return THR_ERR_BADARG;
  if (imass != 1 && imass != 3) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  THR_TRY(c->ensure_w64(8));
  THR_TRY(c->use_links(nullptr));
  THR_TRY(c->upload_spinor(c->w64[0], Phi));
  const int niterc = c->g.ls * c->g.v3;  // params.F90:57
  int rc = congrad_o_dev(c, c->w64[0], c->w64[1], res, am, imass, niterc, itercg, iterations);
  if (rc != THR_OK && rc != THR_ERR_MAXITER) return rc;
  THR_TRY(c->download_spinor(X, c->w64[1]));
  const int rs = c->sync();
  return rs ? rs : rc;
}

}  // extern "C"
