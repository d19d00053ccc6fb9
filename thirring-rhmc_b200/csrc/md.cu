// md.cu -- the RHMC layer on device-resident fields: force (force_module.F90),
// hamilton (dwf3d_lib.F90:511-616), initialise_phi_1flavour / initialise_pp
// (evolution.F90:7-111), the leapfrog evolve_theta_pp (evolution.F90:113-179)
// and one trajectory with its Metropolis test (dwf3d_lib.F90:265-323).
//
// Every field of a trajectory (theta, pp, u, Phi, dSdpi, solver vectors)
// stays in HBM; the host only steers: it reads the trajectory-exit draw of
// each MD step and the Hamiltonians.  theta and pp are single precision as
// in the reference; the Hamiltonian sums are accumulated in FP64.
#include <cmath>
#include <cstring>

#include "ctx.h"
#include "md.h"
#include "ms.h"
#include "qmr.h"
#include "rng.h"

namespace thr {

namespace {
constexpr int kThreads = 256;

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double sh[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? sh[threadIdx.x] : 0.0;
  if (w == 0) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

// force_module.F90:102-109: antiperiodic sign on the last t-slice, + beta*Nf*theta
__global__ void k_force_finish(double* dS, const float* theta, Geom g, int ibound, float bnf) {
  int n = g.v3 * 3;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int site = i % g.v3, mu = i / g.v3;
    double v = dS[i];
    if (ibound == -1 && mu == 2) {
      int x, y, t;
      site_coords(g, site, x, y, t);
      if (t == g.lt - 1) v = -v;
    }
    dS[i] = v + (double)__fmul_rn(bnf, theta[i]);
  }
}

// pp = pp - real(c*dSdpi): c = 0.5*dt or dt in single, product in double, rounded (evolution.F90:142,170,173)
__global__ void k_pp_kick(float* pp, const double* dS, float c, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    pp[i] = __fsub_rn(pp[i], (float)((double)c * dS[i]));
}
// thetat = thetat + dt*pp (evolution.F90:157), single precision, no contraction
__global__ void k_theta_drift(float* th, const float* pp, float dt, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    th[i] = __fadd_rn(th[i], __fmul_rn(dt, pp[i]));
}
// sum of squares of a float field in FP64
__global__ void k_sumsq_f(const float* a, int n, double* partials) {
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double v = (double)a[i];
    acc += v * v;
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}
// sum Re(conj(a) b) (dwf3d_lib.F90:594)
__global__ void k_redot(const double2* a, const double2* b, size_t n, double* partials) {
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    acc += a[i].x * b[i].x + a[i].y * b[i].y;
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}
__global__ void k_finish(const double* partials, int np, double* out) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) acc += partials[i];
  acc = block_sum(acc);
  if (threadIdx.x == 0) *out = acc;
}

// Control block of a captured MD step (at dscal + kScalMd + 8): the exit draw of the step,
// whether it was the last, the OR of its solves' status and the fixed-length flag the host
// sets in pinned memory before each launch
struct MdCtl {
  float ytest;
  int last, status, fixed_last;
};
static_assert(sizeof(MdCtl) <= 3 * sizeof(double), "MdCtl fits its slots");

// counts[k] += the iterations of the multishift just run; status |= its status
__global__ void k_md_count(const MsState* ms, double* counts, int k, MdCtl* ctl) {
  counts[k] += (double)ms->it;
  if (ms->status) ctl->status = ms->status;
}
// the step's closing kick: pp -= c*dSdpi with c = dt/2 on the last step, dt otherwise
// (evolution.F90:166-175); last = the host's fixed-length flag or ytest < proby
__global__ void k_pp_kick_last(float* pp, const double* dS, float dt, float hdt, float proby, int fixed_mode,
                               MdCtl* ctl, int n) {
  const bool last = fixed_mode ? ctl->fixed_last != 0 : ctl->ytest < proby;
  const float c = last ? hdt : dt;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    pp[i] = __fsub_rn(pp[i], (float)((double)c * dS[i]));
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->last = last ? 1 : 0;
}

inline unsigned grid(size_t n) {
  size_t b = (n + kThreads - 1) / kThreads;
  if (b > device_sms() * 4) b = device_sms() * 4;
  return (unsigned)(b ? b : 1);
}
}  // namespace

int md_fields(thr_ctx* c, MdFields* f) {
  const size_t n = c->n4();
  const size_t n3 = (size_t)c->g.v3 * 3;
  void *sp, *fp;
  THR_TRY(c->buffer(thr_ctx::B_MD, 4 * n * sizeof(double2), &sp));
  THR_TRY(c->buffer(thr_ctx::B_MDF, 3 * n3 * sizeof(float) + n3 * sizeof(double) + 64, &fp));
  f->Phi = (double2*)sp;
  f->X2 = f->Phi + n;
  f->Xr = f->X2 + n;
  f->R = f->Xr + n;
  f->theta = (float*)fp;
  f->thetat = f->theta + n3;
  f->pp = f->thetat + n3;
  f->dS = (double*)(f->pp + n3 + (n3 & 1));
  return THR_OK;
}

static int reduce_to_host(thr_ctx* c, int np, double* out) {
  k_finish<<<1, 1024, 0, c->st>>>(c->partials, np, c->dscal + kScalHamSum);
  THR_CUDA(cudaMemcpyAsync(c->hscal + kScalHamSum, c->dscal + kScalHamSum, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  THR_CUDA(cudaStreamSynchronize(c->st));
  *out = c->hscal[kScalHamSum];
  return THR_OK;
}

static int need_rat(thr_ctx* c) { return c->rat.set ? THR_OK : THR_ERR_BADARG; }

// force_module.F90:9-113 on device theta; result in f->dS
int force_dev(thr_ctx* c, MdFields* f, const float* theta, float res1, float am, int imass) {
  THR_TRY(need_rat(c));
  const size_t n = c->n4();
  const size_t n3 = (size_t)c->g.v3 * 3;
  auto& R = c->rat;
  const int ng = R.ndiagg;
  const int sp = c->spmd;
  const float One = 1.0f;
  int it = 0;
  // iteration sums: on the host, or -- inside a captured MD step -- on the device
  auto count = [&](int k) {
    if (c->md_capture)
      k_md_count<<<1, 1, 0, c->st>>>(reinterpret_cast<const MsState*>(c->dscal), c->dscal + kScalMd, k,
                                     reinterpret_cast<MdCtl*>(c->dscal + kScalMd + 8));
    else
      c->md_counts[k] += it;
  };
  THR_CUDA(cudaMemsetAsync(f->dS, 0, n3 * sizeof(double), c->st));
  THR_CUDA(cudaMemcpyAsync(f->X2, f->Phi, n * sizeof(double2), cudaMemcpyDeviceToDevice, c->st));
  THR_TRY(qmrherm_dev(c, f->X2, f->Xr, res1, &it, One, 1, R.anum4g.data(), R.aden4g.data(), ng, 1, sp, nullptr,
                      f->dS, c->max_qmr_iters));
  count(1);  // ancgpv
  THR_CUDA(cudaMemcpyAsync(f->X2, f->Xr, n * sizeof(double2), cudaMemcpyDeviceToDevice, c->st));
  THR_TRY(qmrherm_dev(c, f->X2, f->Xr, res1, &it, am, imass, R.bnum2g.data(), R.bden2g.data(), ng, 0, sp, nullptr,
                      f->dS, c->max_qmr_iters));
  count(0);  // ancg
  THR_CUDA(cudaMemcpyAsync(f->X2, f->Xr, n * sizeof(double2), cudaMemcpyDeviceToDevice, c->st));
  THR_TRY(qmrherm_dev(c, f->X2, f->Xr, res1, &it, am, imass, R.anum2g.data(), R.aden2g.data(), ng, 2, sp, nullptr,
                      f->dS, c->max_qmr_iters));
  count(2);  // ancgf
  THR_TRY(qmrherm_dev(c, f->X2, f->Xr, res1, &it, One, 1, R.anum4g.data(), R.aden4g.data(), ng, 3, sp, nullptr,
                      f->dS, c->max_qmr_iters));
  count(3);  // ancgfpv
  const float bnf = c->p.beta * 1.0f;  // beta*Nf, Nf = 1 (params.F90:19)
  k_force_finish<<<grid(n3), kThreads, 0, c->st>>>(f->dS, theta, c->g, c->p.ibound, bnf);
  return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
}

// dwf3d_lib.F90:511-616 with the context's current links
int hamilton_dev(thr_ctx* c, MdFields* f, const float* theta, const float* pp, float res2, float am, int imass,
                 double* h, double* hg, double* hp, double* s) {
  THR_TRY(need_rat(c));
  const size_t n = c->n4();
  const int n3 = c->g.v3 * 3;
  double spp, sth;
  k_sumsq_f<<<grid(n3), kThreads, 0, c->st>>>(pp, n3, c->partials);
  THR_TRY(reduce_to_host(c, (int)grid(n3), &spp));
  k_sumsq_f<<<grid(n3), kThreads, 0, c->st>>>(theta, n3, c->partials);
  THR_TRY(reduce_to_host(c, (int)grid(n3), &sth));
  *hp = 0.5 * spp;
  *hg = 0.5 * 1.0 * (double)c->p.beta * sth;
  auto& R = c->rat;
  int it = 0;
  THR_CUDA(cudaMemcpyAsync(f->R, f->Phi, n * sizeof(double2), cudaMemcpyDeviceToDevice, c->st));
  THR_TRY(qmrherm_dev(c, f->R, f->Xr, res2, &it, 1.0f, 1, R.anum4.data(), R.aden4.data(), R.ndiag, 0, c->action_sp,
                      nullptr, nullptr, c->max_qmr_iters));
  c->md_counts[5] += it;  // ancghpv
  if (it >= c->max_qmr_iters) return THR_ERR_MAXITER;  // check_qmr_iterations: dwf3d_lib.F90:860-881
  THR_CUDA(cudaMemcpyAsync(f->R, f->Xr, n * sizeof(double2), cudaMemcpyDeviceToDevice, c->st));
  THR_TRY(qmrherm_dev(c, f->R, f->Xr, res2, &it, am, imass, R.bnum2.data(), R.bden2.data(), R.ndiag, 0,
                      c->action_sp, nullptr, nullptr, c->max_qmr_iters));
  c->md_counts[4] += it;  // ancgh
  if (it >= c->max_qmr_iters) return THR_ERR_MAXITER;
  k_redot<<<grid(n), kThreads, 0, c->st>>>(f->R, f->Xr, n, c->partials);
  double hf;
  THR_TRY(reduce_to_host(c, (int)grid(n), &hf));
  *h = *hg + *hp + hf;
  *s = *hg + hf;
  return THR_OK;
}

// evolution.F90:7-75 (Phi from a fresh Gaussian R) with the current links
int initialise_phi_dev(thr_ctx* c, MdFields* f, float am, int imass) {
  THR_TRY(need_rat(c));
  const size_t n = c->n4();
  auto& R = c->rat;
  THR_TRY(rng_phi_draw(c, f->R));
  int it = 0;
  THR_TRY(qmrherm_dev(c, f->R, f->Xr, c->rescga, &it, am, imass, R.anum4.data(), R.aden4.data(), R.ndiag, 0,
                      c->action_sp, nullptr, nullptr, c->max_qmr_iters));
  c->md_counts[6] += it;  // ancgpf
  THR_CUDA(cudaMemcpyAsync(f->R, f->Xr, n * sizeof(double2), cudaMemcpyDeviceToDevice, c->st));
  THR_TRY(qmrherm_dev(c, f->R, f->Xr, c->rescga, &it, 1.0f, 1, R.bnum4.data(), R.bden4.data(), R.ndiag, 0,
                      c->action_sp, nullptr, nullptr, c->max_qmr_iters));
  c->md_counts[7] += it;  // ancgpfpv
  THR_CUDA(cudaMemcpyAsync(f->Phi, f->Xr, n * sizeof(double2), cudaMemcpyDeviceToDevice, c->st));
  return THR_OK;
}

namespace {
// One MD step -- drift, coef, force (four multishift solves, each batch loop a WHILE
// node), the exit draw at site (1,1,1), the closing kick -- captured once and replayed.
struct MdGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  MdFields f{};
  float dt = 0.f, res = 0.f, am = 0.f, proby = 0.f, am3 = 0.f, beta = 0.f;
  int imass = 0, fixed_mode = 0, spmd = -1;
  unsigned long long gen = ~0ull;
  bool failed = false;  // a capture failed for this key: run host-driven
  void release() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
};
constexpr int kFixedLastSlot = 1000;  // hiscal slot the step graph copies its fixed-length flag from

bool md_same(const MdGraph& G, const thr_ctx* c, const MdFields* f, float dt, float res, float am, int imass,
             float proby, int fixed_mode) {
  return G.f.Phi == f->Phi && G.f.thetat == f->thetat && G.f.pp == f->pp && G.f.dS == f->dS && G.f.X2 == f->X2 &&
         G.f.Xr == f->Xr && G.dt == dt && G.res == res && G.am == am && G.imass == imass && G.proby == proby &&
         G.fixed_mode == fixed_mode && G.gen == c->buf_gen && G.am3 == c->p.am3 && G.beta == c->p.beta &&
         G.spmd == c->spmd;
}

// captures the step into G (c->st in capture mode); on failure the capture is discarded
int md_capture_step(thr_ctx* c, MdGraph& G, MdFields* f, float dt, float res, float am, int imass, float proby,
                    int fixed_mode) {
  const int n3 = c->g.v3 * 3;
  const float hdt = 0.5f * dt;
  MdCtl* ctl = reinterpret_cast<MdCtl*>(c->dscal + kScalMd + 8);
  G.release();
  THR_CUDA(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
  c->md_capture = true;
  c->ms_tmpl_next = 0;
  int rc = THR_OK;
  if (cudaMemsetAsync(c->dscal + kScalMd, 0, 8 * sizeof(double) + sizeof(MdCtl), c->st) != cudaSuccess ||
      cudaMemcpyAsync(&ctl->fixed_last, c->hiscal + kFixedLastSlot, sizeof(int), cudaMemcpyHostToDevice, c->st) !=
          cudaSuccess)
    rc = THR_ERR_CUDA;
  if (!rc) {
    k_theta_drift<<<grid(n3), kThreads, 0, c->st>>>(f->thetat, f->pp, dt, n3);
    rc = c->coef_dev(f->thetat);
  }
  if (!rc) rc = force_dev(c, f, f->thetat, res, am, imass);
  if (!rc) rc = rng_rano_site(c, 1, 1, 1, &ctl->ytest, nullptr);  // evolution.F90:146
  if (!rc) k_pp_kick_last<<<grid(n3), kThreads, 0, c->st>>>(f->pp, f->dS, dt, hdt, proby, fixed_mode, ctl, n3);
  c->md_capture = false;
  cudaGraph_t g = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(c->st, &g);
  if (!rc && ce == cudaSuccess && g) {
    G.graph = g;
    if (cudaGraphInstantiate(&G.exec, G.graph, cudaGraphInstantiateFlagUseNodePriority) != cudaSuccess)
      rc = THR_ERR_CUDA;
  } else {
    if (g) cudaGraphDestroy(g);
    if (!rc) rc = THR_ERR_CUDA;
  }
  if (rc) {
    G.release();
    cudaGetLastError();
    return rc;
  }
  G.f = *f;
  G.dt = dt; G.res = res; G.am = am; G.imass = imass; G.proby = proby; G.fixed_mode = fixed_mode;
  G.gen = c->buf_gen; G.am3 = c->p.am3; G.beta = c->p.beta; G.spmd = c->spmd;
  return THR_OK;
}
}  // namespace

void md_graph_release(thr_ctx* c) {
  if (c->md_graph) {
    static_cast<MdGraph*>(c->md_graph)->release();
    delete static_cast<MdGraph*>(c->md_graph);
    c->md_graph = nullptr;
  }
}

// evolution.F90:113-179 on f->thetat / f->pp; links follow thetat.  The first MD step
// runs host-driven (it sizes every buffer and settles the autotuner); the others replay
// one captured graph of the step: one launch and one synchronisation per step.
int evolve_dev(thr_ctx* c, MdFields* f, int iterl, float dt, float res, float am, int imass, int fixed_steps,
               int* itot) {
  const int n3 = c->g.v3 * 3;
  THR_TRY(force_dev(c, f, f->thetat, res, am, imass));
  const float hdt = 0.5f * dt;
  k_pp_kick<<<grid(n3), kThreads, 0, c->st>>>(f->pp, f->dS, hdt, n3);
  const float proby = 1.0f / (float)iterl;
  const int nmax = fixed_steps > 0 ? fixed_steps : 4 * iterl;
  const int fixed_mode = fixed_steps > 0 ? 1 : 0;
  // the step graph needs the site streams (the exit draw on the device), the batched
  // solver and no kernel sampling
  bool graph = c->use_md_graph && c->use_graphs && c->ms_algo == 1 && c->rng.site && !c->prof_on;
  int iter;
  for (iter = 1; iter <= nmax; iter++) {
    if (graph && iter > 1) {
      if (!c->md_graph) c->md_graph = new MdGraph();
      MdGraph& G = *static_cast<MdGraph*>(c->md_graph);
      if (!G.exec || !md_same(G, c, f, dt, res, am, imass, proby, fixed_mode)) {
        if (md_capture_step(c, G, f, dt, res, am, imass, proby, fixed_mode) != THR_OK) graph = false;
      }
      if (graph) {
        c->hiscal[kFixedLastSlot] = (fixed_mode && iter == fixed_steps) ? 1 : 0;
        THR_CUDA(cudaGraphLaunch(G.exec, c->st));
        THR_CUDA(cudaMemcpyAsync(c->hscal + kScalMd, c->dscal + kScalMd, 8 * sizeof(double) + sizeof(MdCtl),
                                 cudaMemcpyDeviceToHost, c->st));
        THR_CUDA(cudaStreamSynchronize(c->st));
        for (int k = 0; k < 8; k++) c->md_counts[k] += c->hscal[kScalMd + k];
        const MdCtl* hc = reinterpret_cast<const MdCtl*>(c->hscal + kScalMd + 8);
        if (hc->status) return hc->status;
        if (hc->last) break;
        continue;
      }
    }
    k_theta_drift<<<grid(n3), kThreads, 0, c->st>>>(f->thetat, f->pp, dt, n3);
    THR_TRY(c->coef_dev(f->thetat));
    THR_TRY(force_dev(c, f, f->thetat, res, am, imass));
    float ytest = 0.0f;
    THR_TRY(rng_rano_site(c, 1, 1, 1, nullptr, &ytest));  // evolution.F90:146
    const bool last = fixed_steps > 0 ? (iter == fixed_steps) : (ytest < proby);
    if (last) {
      k_pp_kick<<<grid(n3), kThreads, 0, c->st>>>(f->pp, f->dS, hdt, n3);
      break;
    }
    k_pp_kick<<<grid(n3), kThreads, 0, c->st>>>(f->pp, f->dS, dt, n3);
  }
  if (itot) *itot += iter < nmax ? iter : nmax;
  return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
}

// one pass of dwf3d_lib.F90:265-323 on device theta (f->theta), accepted field left in f->theta
int trajectory_dev(thr_ctx* c, MdFields* f, int iterl, float dt, float am, int imass, int fixed_steps,
                   thr_traj_result* out) {
  const int n3 = c->g.v3 * 3;
  THR_CUDA(cudaMemcpyAsync(f->thetat, f->theta, n3 * sizeof(float), cudaMemcpyDeviceToDevice, c->st));
  THR_TRY(c->coef_dev(f->thetat));
  THR_TRY(initialise_phi_dev(c, f, am, imass));
  THR_TRY(rng_pp_draw(c, f->pp));
  double h0, h1, hg, hp, s0, s1;
  THR_TRY(hamilton_dev(c, f, f->thetat, f->pp, c->rescga, am, imass, &h0, &hg, &hp, &s0));
  int itot = 0;
  THR_TRY(evolve_dev(c, f, iterl, dt, c->rescgg, am, imass, fixed_steps, &itot));
  THR_TRY(hamilton_dev(c, f, f->thetat, f->pp, c->rescga, am, imass, &h1, &hg, &hp, &s1));
  const double dH = h0 - h1;
  const float y = expf((float)dH);  // y = exp(real(dH)) (:304)
  int accept = 1;
  if (dH < 0.0) {
    float x = 0.0f;
    THR_TRY(rng_rano_site(c, 1, 1, 1, nullptr, &x));  // :309
    if (x > y) accept = 0;
  }
  if (accept) THR_CUDA(cudaMemcpyAsync(f->theta, f->thetat, n3 * sizeof(float), cudaMemcpyDeviceToDevice, c->st));
  if (out) {
    out->h0 = h0;
    out->h1 = h1;
    out->dh = dH;
    out->ds = s0 - s1;
    out->accepted = accept;
    out->steps = itot;
    out->y = y;
  }
  return c->sync();
}

}  // namespace thr

using namespace thr;

namespace {
int up_f3(thr_ctx* c, float* dev, const float* host) {
  const size_t n3 = (size_t)c->g.v3 * 3;
  THR_CUDA(cudaMemcpyAsync(c->stage, host, n3 * sizeof(float), cudaMemcpyHostToDevice, c->st));
  from_fortran_f3(c->g, dev, (const float*)c->stage, c->st);
  return THR_OK;
}
int down_f3(thr_ctx* c, float* host, const float* dev) {
  const size_t n3 = (size_t)c->g.v3 * 3;
  to_fortran_f3(c->g, (float*)c->stage, dev, c->st);
  THR_CUDA(cudaMemcpyAsync(host, c->stage, n3 * sizeof(float), cudaMemcpyDeviceToHost, c->st));
  return THR_OK;
}
int down_d3(thr_ctx* c, double* host, const double* dev) {
  const size_t n3 = (size_t)c->g.v3 * 3;
  to_fortran_d3(c->g, (double*)c->stage, dev, c->st);
  THR_CUDA(cudaMemcpyAsync(host, c->stage, n3 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  return THR_OK;
}
void copyv(std::vector<double>& v, const double* a, int n) { v.assign(a, a + n); }
}  // namespace

extern "C" {

int thr_set_remez(thr_ctx* c, int ndiag, const double* anum2, const double* aden2, const double* bnum2,
                  const double* bden2, const double* anum4, const double* aden4, const double* bnum4,
                  const double* bden4, int ndiagg, const double* anum2g, const double* aden2g, const double* bnum2g,
                  const double* bden2g, const double* anum4g, const double* aden4g, const double* bnum4g,
                  const double* bden4g) {
  if (!c || ndiag < 1 || ndiagg < 1 || ndiag > 64 || ndiagg > 64) return THR_ERR_BADARG;
  if (ndiag > c->p.ndiag || ndiagg > c->p.ndiag) return THR_ERR_BADSHAPE;
  auto& R = c->rat;
  R.ndiag = ndiag;
  R.ndiagg = ndiagg;
  copyv(R.anum2, anum2, ndiag + 1); copyv(R.aden2, aden2, ndiag);
  copyv(R.bnum2, bnum2, ndiag + 1); copyv(R.bden2, bden2, ndiag);
  copyv(R.anum4, anum4, ndiag + 1); copyv(R.aden4, aden4, ndiag);
  copyv(R.bnum4, bnum4, ndiag + 1); copyv(R.bden4, bden4, ndiag);
  copyv(R.anum2g, anum2g, ndiagg + 1); copyv(R.aden2g, aden2g, ndiagg);
  copyv(R.bnum2g, bnum2g, ndiagg + 1); copyv(R.bden2g, bden2g, ndiagg);
  copyv(R.anum4g, anum4g, ndiagg + 1); copyv(R.aden4g, aden4g, ndiagg);
  copyv(R.bnum4g, bnum4g, ndiagg + 1); copyv(R.bden4g, bden4g, ndiagg);
  R.set = true;
  return THR_OK;
}

int thr_set_residuals(thr_ctx* c, float rescga, float rescgg, int spmd, int max_qmr_iters) {
  if (!c || spmd < 0 || spmd > 3) return THR_ERR_BADARG;
  c->rescga = rescga;
  c->rescgg = rescgg;
  c->spmd = spmd;
  if (max_qmr_iters > 0) c->max_qmr_iters = max_qmr_iters;
  return THR_OK;
}

int thr_set_action_precision(thr_ctx* c, int precision) {
  if (!c || (precision != THR_FP64 && precision != THR_MIXED_FP32 && precision != THR_MIXED_BF16))
    return THR_ERR_BADARG;
  c->action_sp = precision;
  return THR_OK;
}

int thr_force(thr_ctx* c, const double* Phi, float res1, float am, int imass, const float* theta, double* dSdpi) {
  if (!c || !Phi || !theta || !dSdpi) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  MdFields f;
  THR_TRY(md_fields(c, &f));
  THR_TRY(c->use_links(nullptr));
  THR_TRY(c->upload_spinor(f.Phi, Phi));
  THR_TRY(up_f3(c, f.thetat, theta));
  THR_TRY(force_dev(c, &f, f.thetat, res1, am, imass));
  THR_TRY(down_d3(c, dSdpi, f.dS));
  return c->sync();
}

int thr_hamilton(thr_ctx* c, const double* Phi, double* h, double* hg, double* hp, double* s, float res2, float am,
                 int imass, const float* theta, const float* pp) {
  if (!c || !Phi || !h || !hg || !hp || !s || !theta || !pp) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  MdFields f;
  THR_TRY(md_fields(c, &f));
  THR_TRY(c->use_links(nullptr));
  THR_TRY(c->upload_spinor(f.Phi, Phi));
  THR_TRY(up_f3(c, f.thetat, theta));
  THR_TRY(up_f3(c, f.pp, pp));
  THR_TRY(hamilton_dev(c, &f, f.thetat, f.pp, res2, am, imass, h, hg, hp, s));
  return c->sync();
}

int thr_initialise_phi(thr_ctx* c, double* Phi, float am, int imass) {
  if (!c || !Phi) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  MdFields f;
  THR_TRY(md_fields(c, &f));
  THR_TRY(c->use_links(nullptr));
  THR_TRY(initialise_phi_dev(c, &f, am, imass));
  THR_TRY(c->download_spinor(Phi, f.Phi));
  return c->sync();
}

int thr_initialise_pp(thr_ctx* c, float* pp) {
  if (!c || !pp) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  MdFields f;
  THR_TRY(md_fields(c, &f));
  THR_TRY(rng_pp_draw(c, f.pp));
  THR_TRY(down_f3(c, pp, f.pp));
  return c->sync();
}

int thr_evolve_theta_pp(thr_ctx* c, int iterl, float dt, float* pp, const double* Phi, float res, float am, int imass,
                        int* itot, float* theta, double* u, double* dSdpi, int fixed_steps) {
  if (!c || !pp || !Phi || !theta || iterl < 1) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  MdFields f;
  THR_TRY(md_fields(c, &f));
  THR_TRY(c->upload_spinor(f.Phi, Phi));
  THR_TRY(up_f3(c, f.thetat, theta));
  THR_TRY(up_f3(c, f.pp, pp));
  THR_TRY(c->coef_dev(f.thetat));
  int it = itot ? *itot : 0;
  THR_TRY(evolve_dev(c, &f, iterl, dt, res, am, imass, fixed_steps, &it));
  if (itot) *itot = it;
  THR_TRY(down_f3(c, theta, f.thetat));
  THR_TRY(down_f3(c, pp, f.pp));
  if (dSdpi) THR_TRY(down_d3(c, dSdpi, f.dS));
  if (u) {
    to_fortran_links(c->g, c->stage, c->u64, c->st);
    THR_CUDA(cudaMemcpyAsync(u, c->stage, c->nfl() * sizeof(double2), cudaMemcpyDeviceToHost, c->st));
  }
  return c->sync();
}

int thr_trajectory(thr_ctx* c, float* theta, int iterl, float dt, float am, int imass, int fixed_steps,
                   thr_traj_result* out) {
  if (!c || !theta || iterl < 1) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  MdFields f;
  THR_TRY(md_fields(c, &f));
  THR_TRY(up_f3(c, f.theta, theta));
  THR_TRY(trajectory_dev(c, &f, iterl, dt, am, imass, fixed_steps, out));
  THR_TRY(down_f3(c, theta, f.theta));
  return c->sync();
}

int thr_md_counters(thr_ctx* c, double* counts8, int reset) {
  if (!c) return THR_ERR_BADARG;
  if (counts8) memcpy(counts8, c->md_counts, sizeof(c->md_counts));
  if (reset) memset(c->md_counts, 0, sizeof(c->md_counts));
  return THR_OK;
}

}  // extern "C"
