// measure.cu -- the noisy psibarpsi estimator (measure_module.F90:142-670)
// on the device, with every noise's solves batched into one congrad.
//
// The reference draws two Gaussian noise fields per noise (gauss0(ps),
// gauss0(pt)), and for each source spin solves M^dagger M X = M^dagger xi for
// a domain-wall source xi on the wall s = 1 (from ps) or s = Ls (from pt),
// one congrad call at a time, the source doubling as the initial guess
// (vector::X is xi).  Congrad never touches the random numbers, so here all
// draws come first, then all sources are built and solved together by the
// batched congrad (one persistent stencil launch per operation for all
// right-hand sides), and one kernel contracts every solution with its noise.
//
//   measure_shamir (:170-423): 2 source spins per wall, the solution on the
//     opposite wall contracted directly.
//   measure_wilson (:431-670): 4 source spins per wall; the wall slice of the
//     solution is first replaced by DWilson(P xi, -am3) - P xi, P = P+
//     (spins 1,2) at s = Ls, P- (spins 3,4) at s = 1 (:523-527, :576-580).
//
// Sums over the lattice are FP64 complex (block partials in a fixed order,
// summed on the host in solve order); the scalar results follow the
// reference's kinds (pbp real(dp), psibarpsi and susclsing default real).
#include <algorithm>
#include <vector>

#include "ctx.h"
#include "overlap.h"
#include "rng.h"

namespace thr {

namespace {

struct MeasSolve {
  int noise;    // eta field: 2 * inoise + (0: ps, 1: pt)
  int s_src, d_src;
  double sign;  // -1 for the gamma_5 sources of imass = 5 (:229-236)
  int s_c, d_c;  // contraction wall and spin
  int post;      // 0 none, 1: DWilson on P+ slice, 2: DWilson on P- slice
  int part;      // psibarpsi1 (0) or psibarpsi2 (1)
};

constexpr int kMeasThreads = 256;

// the reference's solve order of one noise (0-based spins and walls)
std::vector<MeasSolve> solves_of_noise(int n, int ls, int imass, int kernel_meas) {
  std::vector<MeasSolve> v;
  if (kernel_meas == 0) {
    for (int i = 0; i < 2; i++) {
      if (imass != 5) {
        v.push_back({2 * n, 0, i, 1.0, ls - 1, i, 0, 0});
        v.push_back({2 * n + 1, ls - 1, i + 2, 1.0, 0, i + 2, 0, 1});
      } else {
        v.push_back({2 * n, 0, i, -1.0, 0, i + 2, 0, 0});
        v.push_back({2 * n + 1, ls - 1, i + 2, -1.0, ls - 1, i, 0, 1});
      }
    }
  } else {
    for (int i = 0; i < 4; i++) v.push_back({2 * n, 0, i, 1.0, ls - 1, i, 1, 0});
    for (int i = 0; i < 4; i++) v.push_back({2 * n + 1, ls - 1, i, 1.0, 0, i, 2, 1});
  }
  return v;
}

// xi_j = sign * cmplx(eta_1, eta_2) on (s_src, spin d_src), zero elsewhere
// (the fields are cleared beforehand); grid (site blocks, solves)
__global__ void k_meas_source(double2* __restrict__ X, const float* __restrict__ eta, const MeasSolve* __restrict__ sv,
                              Geom g, size_t n4) {
  const int site = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (site >= g.v3) return;
  const MeasSolve m = sv[j];
  const float* e = eta + (size_t)m.noise * 2 * g.v3;
  X[(size_t)j * n4 + sidx(g, m.s_src, site, m.d_src)] =
      make_double2(m.sign * (double)e[site], m.sign * (double)e[g.v3 + site]);
}

__device__ __forceinline__ double2 wall_value(const double2* __restrict__ X, const double2* __restrict__ u,
                                              const Geom& g, const MeasSolve& m, int site, double dgw) {
  if (m.post == 0) return X[sidx(g, m.s_c, site, m.d_c)];
  // islice(d) = X(s_c, ., d) for d in the projector's spins, else 0
  const int d0 = m.post == 1 ? 0 : 2;
  auto is = [&](int st, int d) -> double2 {
    return (d >= d0 && d < d0 + 2) ? X[sidx(g, m.s_c, st, d)] : make_double2(0.0, 0.0);
  };
  int x, y, t;
  site_coords(g, site, x, y, t);
  const Nbr nb = neighbours(g, site, x, y, t);
  const int d = m.d_c;
  double2 out = dgw * is(site, d);  // DWilson: Phi = diag * R (dirac.F90:191-192)
#pragma unroll
  for (int mu = 0; mu < 3; mu++) {
    const double2 U = u[(size_t)mu * g.v3 + site];
    const double2 Ub = cconj(u[(size_t)mu * g.v3 + nb.b[mu]]);
    const GammaEntry ge = gamma_entry(mu, d);
    const double2 A = cmul(U, is(nb.f[mu], d)), B = cmul(Ub, is(nb.b[mu], d));
    const double2 Ag = cmul(U, is(nb.f[mu], ge.gin)), Bg = cmul(Ub, is(nb.b[mu], ge.gin));
    out = (out - 0.5 * (A + B)) + gmul<double2, double>(ge, Ag - Bg);  // dirac.F90:205-217
  }
  return out - is(site, d);  // oslice = oslice - islice
}

// partials[j * nblk + block] = sum over the block's sites of conj(eta) * wall value
__global__ void __launch_bounds__(kMeasThreads) k_meas_contract(const double2* __restrict__ X,
                                                                 const float* __restrict__ eta,
                                                                 const double2* __restrict__ u,
                                                                 const MeasSolve* __restrict__ sv, Geom g, size_t n4,
                                                                 double dgw, double2* __restrict__ partials) {
  const int site = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  const MeasSolve m = sv[j];
  double2 acc = make_double2(0.0, 0.0);
  if (site < g.v3) {
    const float* e = eta + (size_t)m.noise * 2 * g.v3;
    const double2 eta_c = make_double2((double)e[site], (double)e[g.v3 + site]);
    acc = cjmul(eta_c, wall_value(X + (size_t)j * n4, u, g, m, site, dgw));
  }
  __shared__ double2 sh[kMeasThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    acc.x += __shfl_down_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_down_sync(0xffffffffu, acc.y, o);
  }
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double2 s = sh[0];
    for (int w = 1; w < kMeasThreads / 32; w++) s = s + sh[w];
    partials[(size_t)j * gridDim.x + blockIdx.x] = s;
  }
}

// propagator sources on the wall s = 1 (0-based s = 0), spin d: a point source at
// storage site `site` (site >= 0) or a wall on the time slice t (site < 0), value v
__global__ void k_prop_source(double2* X, Geom g, size_t n4, int d, int site, int t, double v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.v3) return;
  if (site >= 0) {
    if (i == 0) X[sidx(g, 0, site, d)] = make_double2(v, 0.0);
    return;
  }
  int x, y, tt;
  site_coords(g, i, x, y, tt);
  if (tt == t) X[sidx(g, 0, i, d)] = make_double2(v, 0.0);
}

// the two walls of a propagator: W[0..1][site] = X(s = 1, spins 1,2),
// W[2..3][site] = X(s = Ls, spins 3,4) (storage site order)
__global__ void k_prop_walls(double2* W, const double2* X, Geom g) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.v3) return;
  for (int k = 0; k < 2; k++) {
    W[(size_t)k * g.v3 + i] = X[sidx(g, 0, i, k)];
    W[(size_t)(2 + k) * g.v3 + i] = X[sidx(g, g.ls - 1, i, 2 + k)];
  }
}
}  // namespace

// Solves the propagators of `src` (one wall-s = 1 source each, built by the caller
// on X) as measure_module.F90:811-826 does: Phi = M^dagger xi, initial guess
// M^dagger Phi, congrad; returns the two walls of every solution on the host
// (W: per solve 4 x V3 double2) and the iteration counts.
static int prop_walls(thr_ctx* c, double2* X, int nsol, float res, float am, int imass, int precision,
               std::vector<double2>& W, int* its) {
  const Geom& g = c->g;
  const size_t n4 = c->n4();
  double2 *Phi = nullptr, *Wd = nullptr;
  int rc = THR_OK;
  if (cudaMalloc(&Phi, sizeof(double2) * n4 * nsol) != cudaSuccess ||
      cudaMalloc(&Wd, sizeof(double2) * 4 * (size_t)g.v3 * nsol) != cudaSuccess)
    rc = THR_ERR_NOMEM;
  for (int j = 0; !rc && j < nsol; j++) {
    rc = launch_dslash<double2>(g, c->p.kernel, true, Phi + j * n4, X + j * n4, c->u64, am, imass, c->p.am3, c->st,
                                nullptr);
    if (!rc)
      rc = launch_dslash<double2>(g, c->p.kernel, true, X + j * n4, Phi + j * n4, c->u64, am, imass, c->p.am3,
                                  c->st, nullptr);
  }
  int outer = 0;
  if (!rc) rc = thr_congrad_multi_dev(c, Phi, X, nsol, res, am, imass, precision, its, &outer);
  if (rc == THR_ERR_MAXITER) rc = THR_OK;  // congrad only writes a notice at niterc
  const unsigned nb = (unsigned)((g.v3 + 255) / 256);
  for (int j = 0; !rc && j < nsol; j++) k_prop_walls<<<nb, 256, 0, c->st>>>(Wd + (size_t)j * 4 * g.v3, X + j * n4, g);
  if (!rc) {
    W.resize((size_t)4 * g.v3 * nsol);
    if (cudaMemcpyAsync(W.data(), Wd, sizeof(double2) * W.size(), cudaMemcpyDeviceToHost, c->st) != cudaSuccess ||
        cudaStreamSynchronize(c->st) != cudaSuccess)
      rc = THR_ERR_CUDA;
  }
  cudaFree(Phi);
  cudaFree(Wd);
  return rc;
}

}  // namespace thr

using namespace thr;

extern "C" {

int thr_measure(thr_ctx* c, int kernel_meas, float res, float am, int imass, int knoise, int precision,
                float* psibarpsi, float* susclsing, float* aviter, double* parts, int* itercg) {
  if (!c || !psibarpsi || !susclsing || !aviter || knoise < 1) return THR_ERR_BADARG;
  if (kernel_meas == 2) {  // measure_wilsonKDDW, FP64 only
    if (precision != THR_FP64) return THR_ERR_UNSUPPORTED;
    if (!c->links_ok || !c->rng.ready) return THR_ERR_BADARG;
    cudaSetDevice(c->dev);
    return measure_ow(c, res, am, imass, knoise, psibarpsi, susclsing, aviter, parts, itercg);
  }
  if (kernel_meas != 0 && kernel_meas != 1) return THR_ERR_BADARG;
  if (imass != 1 && imass != 3 && imass != 5) return THR_ERR_BADARG;
  if (kernel_meas == 1 && imass == 5) return THR_ERR_UNSUPPORTED;  // measure_wilson has no imass 5 branch
  if (c->p.kernel == 1 && imass == 5) return THR_ERR_UNSUPPORTED;
  if (!c->links_ok || !c->rng.ready) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  const Geom& g = c->g;
  const size_t n4 = c->n4();
  const int per_noise = kernel_meas == 0 ? 4 : 8;

  // all noise draws first, in the reference's order: gauss0(ps), gauss0(pt) per noise
  float* eta = nullptr;
  THR_CUDA(cudaMalloc(&eta, sizeof(float) * 2 * (size_t)g.v3 * 2 * knoise));
  std::vector<MeasSolve> all;
  for (int n = 0; n < knoise; n++) {
    for (int w = 0; w < 2; w++) {
      int rc = rng_gauss_dev(c, -1.0f, eta + (size_t)(2 * n + w) * 2 * g.v3);
      if (rc) { cudaFree(eta); return rc; }
    }
    for (const MeasSolve& m : solves_of_noise(n, g.ls, imass, kernel_meas)) all.push_back(m);
  }
  const int nsolve = (int)all.size();

  // solves per batch: the batched congrad holds 12 FP64 fields per right-hand side
  const size_t budget = (size_t)16 << 30;
  int chunk = (int)std::max<size_t>(1, budget / (12 * n4 * sizeof(double2)) / per_noise) * per_noise;
  chunk = std::min(chunk, nsolve);
  const unsigned nblk = (unsigned)((g.v3 + kMeasThreads - 1) / kMeasThreads);
  double2 *Phi = nullptr, *X = nullptr, *part = nullptr;
  MeasSolve* sv = nullptr;
  int rc = THR_OK;
  if (cudaMalloc(&Phi, sizeof(double2) * n4 * chunk) != cudaSuccess ||
      cudaMalloc(&X, sizeof(double2) * n4 * chunk) != cudaSuccess ||
      cudaMalloc(&part, sizeof(double2) * nblk * chunk) != cudaSuccess ||
      cudaMalloc(&sv, sizeof(MeasSolve) * nsolve) != cudaSuccess)
    rc = THR_ERR_NOMEM;
  std::vector<int> its(nsolve, 0);
  std::vector<double2> hpart((size_t)nblk * nsolve);
  if (!rc && cudaMemcpyAsync(sv, all.data(), sizeof(MeasSolve) * nsolve, cudaMemcpyHostToDevice, c->st) != cudaSuccess)
    rc = THR_ERR_CUDA;
  const double dgw = (double)(3.0f + (-c->p.am3));  // DWilson(…, -am3): diag = (3.0 + mass) in default real
  for (int j0 = 0; !rc && j0 < nsolve; j0 += chunk) {
    const int nj = std::min(chunk, nsolve - j0);
    if (cudaMemsetAsync(X, 0, sizeof(double2) * n4 * nj, c->st) != cudaSuccess) { rc = THR_ERR_CUDA; break; }
    k_meas_source<<<dim3(nblk, nj), kMeasThreads, 0, c->st>>>(X, eta, sv + j0, g, n4);
    // Phi = M^dagger xi with the measurement kernel (dslashd_shamir / dslashd_wilson, :246, :507)
    for (int j = 0; !rc && j < nj; j++)
      rc = launch_dslash<double2>(g, kernel_meas, true, Phi + (size_t)j * n4, X + (size_t)j * n4, c->u64, am, imass,
                                  c->p.am3, c->st, nullptr);
    if (rc) break;
    // congrad on the generation kernel, the source as initial guess
    int outer = 0;
    rc = thr_congrad_multi_dev(c, Phi, X, nj, res, am, imass, precision, its.data() + j0, &outer);
    if (rc == THR_ERR_MAXITER) rc = THR_OK;  // congrad only writes a notice at niterc (measure_module.F90:124-135)
    if (rc) break;
    k_meas_contract<<<dim3(nblk, nj), kMeasThreads, 0, c->st>>>(X, eta, c->u64, sv + j0, g, n4, dgw, part);
    if (cudaMemcpyAsync(hpart.data() + (size_t)j0 * nblk, part, sizeof(double2) * nblk * nj, cudaMemcpyDeviceToHost,
                        c->st) != cudaSuccess ||
        cudaStreamSynchronize(c->st) != cudaSuccess)
      rc = THR_ERR_CUDA;
  }
  cudaFree(Phi);
  cudaFree(X);
  cudaFree(part);
  cudaFree(sv);
  cudaFree(eta);
  if (rc) return rc;
  if (cudaPeekAtLastError() != cudaSuccess) return THR_ERR_CUDA;

  // the reference's scalar arithmetic (measure_module.F90:336-421)
  const double kvol = (double)g.v3;
  std::vector<double> pbp(knoise);
  long long iter = 0;
  for (int n = 0; n < knoise; n++) {
    double2 acc[2] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
    for (int k = 0; k < per_noise; k++) {
      const int j = n * per_noise + k;
      double2 s = make_double2(0.0, 0.0);
      for (unsigned b = 0; b < nblk; b++) s = s + hpart[(size_t)j * nblk + b];
      acc[all[j].part] = acc[all[j].part] + s;
      iter += its[j];
    }
    double2 p1 = acc[0], p2 = acc[1];
    p1 = make_double2(p1.x / kvol, p1.y / kvol);
    p2 = make_double2(p2.x / kvol, p2.y / kvol);
    if (imass == 3) {  // cmplx(0,-1) * p1, cmplx(0,+1) * p2
      p1 = make_double2(p1.y, -p1.x);
      p2 = make_double2(-p2.y, p2.x);
    } else if (imass == 5) {  // cmplx(0,-1) * both
      p1 = make_double2(p1.y, -p1.x);
      p2 = make_double2(p2.y, -p2.x);
    }
    pbp[n] = p1.x + p2.x;
    if (parts) {
      parts[4 * n + 0] = p1.x; parts[4 * n + 1] = p1.y;
      parts[4 * n + 2] = p2.x; parts[4 * n + 3] = p2.y;
    }
  }
  double sum = 0.0;
  for (int n = 0; n < knoise; n++) sum += pbp[n];
  float pb = (float)sum;
  float sus = 0.0f;
  for (int n = 0; n < knoise; n++) {
    double s = 0.0;
    for (int m = n + 1; m < knoise; m++) s += pbp[n] * pbp[m];
    sus = sus + (float)s;
  }
  pb = pb / (float)knoise;
  sus = (float)(2 * g.v3) * sus / (float)(knoise * (knoise - 1));
  *psibarpsi = pb;
  *susclsing = sus;
  *aviter = (float)iter / (float)(4 * knoise);
  if (itercg) std::copy(its.begin(), its.end(), itercg);
  return THR_OK;
}

// meson(res, itercg, aviter, am, imass), measure_module.F90:684-1085 (SITE_RANDOM,
// nsmear = 0).  Per source three rano draws at site (1,1,1) place a point
// source on the wall s = 1 with spin 3 and 4; the propagators to s = 1 (spins
// 1,2) and s = Ls (spins 3,4) are contracted per time separation from the
// source time.  For imass != 1 the same with -am gives the "n" propagators.
// All solves of one mass go through one batched congrad.
int thr_meson(thr_ctx* c, float res, float am, int imass, int nsource, int precision, double* cpm, double* cmm,
              double* cpmn, double* cmmn, double* chim, int* itercg, float* aviter) {
  if (!c || !cpm || !cmm || !cpmn || !cmmn || !chim || !itercg || !aviter || nsource < 1) return THR_ERR_BADARG;
  if (imass != 1 && imass != 3 && imass != 5) return THR_ERR_BADARG;
  if (c->p.kernel == 1 && imass == 5) return THR_ERR_UNSUPPORTED;
  if (!c->links_ok || !c->rng.ready) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  const Geom& g = c->g;
  const size_t n4 = c->n4();
  const int nsol = 2 * nsource;
  std::vector<int> tsrc(nsource);
  double2* X = nullptr;
  if (cudaMalloc(&X, sizeof(double2) * n4 * nsol) != cudaSuccess) return THR_ERR_NOMEM;
  auto build = [&](std::vector<int>& sites) -> int {
    THR_CUDA(cudaMemsetAsync(X, 0, sizeof(double2) * n4 * nsol, c->st));
    for (int k = 0; k < nsource; k++)
      for (int ids = 0; ids < 2; ids++)
        k_prop_source<<<1, 32, 0, c->st>>>(X + (size_t)(2 * k + ids) * n4, g, n4, 2 + ids, sites[k], 0, 1.0);
    return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
  };
  // source positions: int(ksize * rano) + 1 in default real (:756-758; ksize = Lx for x and y)
  std::vector<int> sites(nsource);
  int rc = THR_OK;
  for (int k = 0; !rc && k < nsource; k++) {
    float r[3];
    for (int q = 0; !rc && q < 3; q++) rc = rng_rano_site(c, 1, 1, 1, nullptr, &r[q]);
    if (rc) break;
    const int ix = (int)((float)g.lx * r[0]), iy = (int)((float)g.lx * r[1]), it = (int)((float)g.lt * r[2]);
    if (ix >= g.lx || iy >= g.ly || it >= g.lt) { rc = THR_ERR_BADSHAPE; break; }
    sites[k] = site_index(g, ix, iy, it);
    tsrc[k] = it;
  }
  std::vector<double2> W, Wn;
  std::vector<int> its(nsol), itsn(nsol, 0);
  if (!rc) rc = build(sites);
  if (!rc) rc = prop_walls(c, X, nsol, res, am, imass, precision, W, its.data());
  if (!rc && imass != 1) {
    rc = build(sites);
    if (!rc) rc = prop_walls(c, X, nsol, res, -am, imass, precision, Wn, itsn.data());
  }
  cudaFree(X);
  if (rc) return rc;
  if (imass == 1) Wn = W;
  // contractions (:900-967): per source, per time separation, sums over x, y, both
  // source spins and the two sink spins, in the Fortran element order
  const int lt = g.lt;
  // natural-order site lists per time slice (x fastest, then y)
  std::vector<std::vector<int>> slice(lt);
  for (int t = 0; t < lt; t++)
    for (int y = 0; y < g.ly; y++)
      for (int x = 0; x < g.lx; x++) slice[t].push_back(site_index(g, x, y, t));
  for (int t = 0; t < lt; t++) {
    cpm[t] = cmm[t] = 0.0;
    cpmn[2 * t] = cpmn[2 * t + 1] = cmmn[2 * t] = cmmn[2 * t + 1] = 0.0;
  }
  const size_t v3 = g.v3;
  for (int k = 0; k < nsource; k++) {
    for (int it = 0; it < lt; it++) {
      const int t = (tsrc[k] + it) % lt;
      double r00 = 0.0, rL = 0.0, c00r = 0.0, c00i = 0.0, cLr = 0.0, cLi = 0.0;
      for (int wall = 0; wall < 2; wall++)       // prop00 (spins 1,2 at s = 1), prop0L (spins 3,4 at s = Ls)
        for (int sp = 0; sp < 2; sp++)           // sink spin (slowest index of the Fortran slice)
          for (int ids = 0; ids < 2; ids++)      // source spin 3, 4
            for (int q : slice[t]) {
              const size_t o = (size_t)(2 * k + ids) * 4 * v3 + (size_t)(2 * wall + sp) * v3 + q;
              const double2 a = W[o], b = Wn[o];
              const double ab2 = a.x * a.x + a.y * a.y;
              const double pr = a.x * b.x + a.y * b.y, pi = a.y * b.x - a.x * b.y;  // a * conj(b)
              if (wall == 0) { r00 += ab2; c00r += pr; c00i += pi; }
              else { rL += ab2; cLr += pr; cLi += pi; }
            }
      cpm[it] += r00;
      cmm[it] += rL;
      cpmn[2 * it] += c00r;
      cpmn[2 * it + 1] += c00i;
      cmmn[2 * it] += cLr;
      cmmn[2 * it + 1] += cLi;
    }
  }
  double ch = 0.0;
  for (int it = 0; it < lt; it++) {
    cpm[it] /= nsource;
    cmm[it] /= nsource;
    for (int q = 0; q < 2; q++) {
      cpmn[2 * it + q] /= nsource;
      cmmn[2 * it + q] /= nsource;
    }
    ch += 2 * (cpm[it] + cmm[it]);
  }
  *chim = ch;
  long long iter = 0;
  for (int j = 0; j < nsol; j++) iter += its[j] + itsn[j];
  *itercg = imass != 1 ? itsn[nsol - 1] : its[nsol - 1];
  *aviter = (float)iter / (float)(2 * nsource);
  return THR_OK;
}

// fermion(res, itercg, aviter, am, imass), measure_module.F90:1100-1376
// (SITE_RANDOM): per source one rano draw picks a time slice; wall sources
// 1/ksize2 (default real) on it at s = 1 with spin 3 and 4;
//   cferm1(t) = sum isign akappa prop0L(x,y,t,d,d),
//   cferm2(t) = sum isign gamval(3,d) prop00(x,y,t,d,gamin(3,d)),
// isign = ibound for sink times before the source time.
int thr_fermion(thr_ctx* c, float res, float am, int imass, int nsource, int precision, double* cferm1,
                double* cferm2, int* itercg, float* aviter) {
  if (!c || !cferm1 || !cferm2 || !itercg || !aviter || nsource < 1) return THR_ERR_BADARG;
  if (imass != 1 && imass != 3 && imass != 5) return THR_ERR_BADARG;
  if (c->p.kernel == 1 && imass == 5) return THR_ERR_UNSUPPORTED;
  if (!c->links_ok || !c->rng.ready) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  const Geom& g = c->g;
  const size_t n4 = c->n4();
  const int nsol = 2 * nsource;
  std::vector<int> tsrc(nsource);
  int rc = THR_OK;
  for (int k = 0; !rc && k < nsource; k++) {
    float r = 0.f;
    rc = rng_rano_site(c, 1, 1, 1, nullptr, &r);
    tsrc[k] = (int)((float)g.lt * r);
    if (!rc && tsrc[k] >= g.lt) rc = THR_ERR_BADSHAPE;
  }
  if (rc) return rc;
  double2* X = nullptr;
  if (cudaMalloc(&X, sizeof(double2) * n4 * nsol) != cudaSuccess) return THR_ERR_NOMEM;
  const double v = (double)(1.0f / (float)(g.lx * g.lx));  // cmplx(1.0,0.0) / ksize2 in default real
  const unsigned nb = (unsigned)((g.v3 + 255) / 256);
  if (cudaMemsetAsync(X, 0, sizeof(double2) * n4 * nsol, c->st) != cudaSuccess) rc = THR_ERR_CUDA;
  for (int k = 0; !rc && k < nsource; k++)
    for (int ids = 0; ids < 2; ids++)
      k_prop_source<<<nb, 256, 0, c->st>>>(X + (size_t)(2 * k + ids) * n4, g, n4, 2 + ids, -1, tsrc[k], v);
  std::vector<double2> W;
  std::vector<int> its(nsol);
  if (!rc) rc = prop_walls(c, X, nsol, res, am, imass, precision, W, its.data());
  cudaFree(X);
  if (rc) return rc;
  const int lt = g.lt;
  std::vector<std::vector<int>> slice(lt);
  for (int t = 0; t < lt; t++)
    for (int y = 0; y < g.ly; y++)
      for (int x = 0; x < g.lx; x++) slice[t].push_back(site_index(g, x, y, t));
  for (int q = 0; q < 2 * lt; q++) cferm1[q] = cferm2[q] = 0.0;
  const size_t v3 = g.v3;
  const double gim[2] = {0.5, -0.5};  // gamval(3, 3:4) = +-i akappa (gammamatrices.F90, mu = 3)
  for (int k = 0; k < nsource; k++) {
    std::vector<double> t1(2 * lt, 0.0), t2(2 * lt, 0.0);
    for (int idd = 0; idd < 2; idd++)
      for (int it = 0; it < lt; it++) {
        const int t = (tsrc[k] + it) % lt;
        const double isign = t >= tsrc[k] ? 1.0 : (double)c->p.ibound;
        double sr = 0.0, si = 0.0;
        for (int q : slice[t]) {  // prop0L(:, :, t, d, d): wall s = Ls, sink spin d = 3 + idd
          const double2 a = W[(size_t)(2 * k + idd) * 4 * v3 + (size_t)(2 + idd) * v3 + q];
          sr += a.x;
          si += a.y;
        }
        t1[2 * it] += isign * 0.5 * sr;
        t1[2 * it + 1] += isign * 0.5 * si;
      }
    for (int idd = 0; idd < 2; idd++)
      for (int it = 0; it < lt; it++) {
        const int t = (tsrc[k] + it) % lt;
        const double isign = t >= tsrc[k] ? 1.0 : (double)c->p.ibound;
        double sr = 0.0, si = 0.0;
        for (int q : slice[t]) {  // prop00(:, :, t, d, gamin(3, d)): wall s = 1, sink spin gamin(3,d) = 1 + idd
          const double2 a = W[(size_t)(2 * k + idd) * 4 * v3 + (size_t)idd * v3 + q];
          sr += a.x;
          si += a.y;
        }
        // isign * (i * gim) * (sr + i si)
        t2[2 * it] += isign * (-gim[idd] * si);
        t2[2 * it + 1] += isign * (gim[idd] * sr);
      }
    for (int q = 0; q < 2 * lt; q++) {
      cferm1[q] += t1[q];
      cferm2[q] += t2[q];
    }
  }
  for (int q = 0; q < 2 * lt; q++) {
    cferm1[q] /= nsource;
    cferm2[q] /= nsource;
  }
  long long iter = 0;
  for (int j = 0; j < nsol; j++) iter += its[j];
  *itercg = its[nsol - 1];
  *aviter = (float)iter / (float)(2 * nsource);
  return THR_OK;
}

}  // extern "C"
