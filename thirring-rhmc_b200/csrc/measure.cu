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
  const Nbr nb = neighbours(g, x, y, t);
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

}  // namespace
}  // namespace thr

using namespace thr;

extern "C" {

int thr_measure(thr_ctx* c, int kernel_meas, float res, float am, int imass, int knoise, int precision,
                float* psibarpsi, float* susclsing, float* aviter, double* parts, int* itercg) {
  if (!c || !psibarpsi || !susclsing || !aviter || knoise < 1) return THR_ERR_BADARG;
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

}  // extern "C"
