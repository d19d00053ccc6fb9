// rng.cu -- random numbers (site_random.f90 / random.f90) and the Gaussian
// draws of gaussian.F90 and evolution.F90.
//
// DRANF (random.f90:87-99) is exact integer arithmetic carried in doubles on
// a 48-bit state in two base-2^24 digits; it equals S <- S*M mod 2^48 with
// M = 2651554*2^24 + 15184245, which is what this file computes in uint64
// (bit-identical, no floating-point rounding involved).  RRANF rounds
// S/2^48 to float; rano is the Numerical Recipes Bays-Durham shuffle over a
// 97-entry table (random.f90:28-58).
//
// Site streams (site_random.f90) are independent per 3D site, so one thread
// advances one site's stream; the global stream (random.f90) is sequential
// and runs on the host.  Box-Muller: log/sin/cos are evaluated by the double
// precision functions and rounded to single; sqrt and the products are
// single precision as in gaussian.F90.
#include <cmath>
#include <cstring>
#include <vector>

#include "ctx.h"
#include "rng.h"

namespace thr {

namespace {
constexpr uint64_t kM = (2651554ULL << 24) + 15184245ULL;
constexpr uint64_t kMask = (1ULL << 48) - 1ULL;
constexpr float kTpi = 2.0f * 3.14159274101257324f;  // 2.0*acos(-1.0) in default real (gaussian.F90:5)

struct Stream {
  uint64_t S;
  float y;
  int idum;
};

__host__ __device__ __forceinline__ float rranf(uint64_t& S) {
  S = (S * kM) & kMask;
  return (float)((double)S * (1.0 / 281474976710656.0));
}

// rano with the table at v (97 entries), state in st
__host__ __device__ __forceinline__ float rano_step(Stream& st, float* v) {
  if (st.idum < 0) {
    st.idum = 1;
    for (int j = 0; j < 97; j++) (void)rranf(st.S);
    for (int j = 0; j < 97; j++) v[j] = rranf(st.S);
    st.y = rranf(st.S);
  }
  int j = 1 + (int)(97.0f * st.y);
  if (j > 97) j = 97;
  if (j < 1) j = 1;
  st.y = v[j - 1];
  const float out = st.y;
  v[j - 1] = rranf(st.S);
  return out;
}

// Box-Muller pair; scale = -1 (gauss0) or -2 (gaussp)
__host__ __device__ __forceinline__ void box_muller(float u1, float u2, float scale, float& ps1, float& ps2) {
  const float lg = (float)log((double)u1);
  const float r = sqrtf(scale * lg);
  const float th = kTpi * u2;
  const float sn = (float)sin((double)th), cs = (float)cos((double)th);
  ps1 = r * sn;
  ps2 = r * cs;
}

// device state: streams[v3], tables[97][v3] (table entry j of site at j*v3+site)
struct TableView {
  float* base;
  int v3, site;
  __device__ __forceinline__ float& operator[](int j) const { return base[(size_t)j * v3 + site]; }
};

// a site's table held in shared memory for the length of a draw: entry j of the block's
// column `col` at base[j * kDrawThreads + col] (one bank per column, conflict-free)
constexpr int kDrawThreads = 64;
struct SmemTable {
  float* base;
  int col;
  __device__ __forceinline__ float& operator[](int j) const { return base[j * kDrawThreads + col]; }
};

template <class View>
__device__ __forceinline__ float rano_dev(Stream& st, View v) {
  if (st.idum < 0) {
    st.idum = 1;
    for (int j = 0; j < 97; j++) (void)rranf(st.S);
    for (int j = 0; j < 97; j++) v[j] = rranf(st.S);
    st.y = rranf(st.S);
  }
  int j = 1 + (int)(97.0f * st.y);
  if (j > 97) j = 97;
  if (j < 1) j = 1;
  st.y = v[j - 1];
  const float out = st.y;
  v[j - 1] = rranf(st.S);
  return out;
}

// init_random: site_random.f90:133-148 (seed_offset :66-73 with ksize = Lx)
__global__ void k_rng_init(Stream* streams, float* tables, Geom g, uint64_t seed) {
  for (int site = blockIdx.x * blockDim.x + threadIdx.x; site < g.v3; site += gridDim.x * blockDim.x) {
    int x, y, t;
    site_coords(g, site, x, y, t);
    const uint64_t off = (uint64_t)x + (uint64_t)g.lx * y + (uint64_t)g.lx * g.lx * t;
    Stream st{(seed + off) & kMask, 0.0f, -1};
    (void)rano_dev(st, TableView{tables, g.v3, site});
    streams[site] = st;
  }
}

// The draw kernels run a site's generator many steps in a row (4 Ls Gaussian pairs for the
// pseudofermion): each step reads and writes one entry of the site's 97-entry shuffle table at
// a random index.  One thread per site copies its table column into shared memory (coalesced:
// the tables are [97][V3]), runs the chain there and copies it back, so the dependent table
// accesses of the chain cost shared-memory latency instead of L2 latency; the arithmetic is
// the same as from global memory, bit for bit.
struct DrawSite {
  float* tab;
  int site;
  bool live;
  __device__ __forceinline__ DrawSite(float* shared_tab, const float* tables, int v3) {
    tab = shared_tab;
    site = blockIdx.x * kDrawThreads + threadIdx.x;
    live = site < v3;
    if (live)
      for (int j = 0; j < 97; j++) tab[j * kDrawThreads + threadIdx.x] = tables[(size_t)j * v3 + site];
  }
  __device__ __forceinline__ SmemTable view() const { return SmemTable{tab, (int)threadIdx.x}; }
  __device__ __forceinline__ void store(float* tables, int v3) const {
    for (int j = 0; j < 97; j++) tables[(size_t)j * v3 + site] = tab[j * kDrawThreads + threadIdx.x];
  }
};

// one gauss0/gaussp call: ps[c][site], c = 0 (sin part), 1 (cos part)
__global__ void __launch_bounds__(kDrawThreads) k_gauss(Stream* streams, float* tables, Geom g, float scale,
                                                        float* ps) {
  __shared__ float tab[97 * kDrawThreads];
  const DrawSite ds(tab, tables, g.v3);
  if (!ds.live) return;
  const int site = ds.site;
  Stream st = streams[site];
  const SmemTable v = ds.view();
  const float u1 = rano_dev(st, v);
  const float u2 = rano_dev(st, v);
  float a, b;
  box_muller(u1, u2, scale, a, b);
  ps[site] = a;
  ps[(size_t)g.v3 + site] = b;
  streams[site] = st;
  ds.store(tables, g.v3);
}

// R(ithird,:,:,:,idirac) = cmplx(gauss0) for idirac = 1..4, ithird = 1..Ls
// in that order (evolution.F90:40-51): 4*Ls gauss0 calls fused per site.
__global__ void __launch_bounds__(kDrawThreads) k_phi_draw(Stream* streams, float* tables, Geom g, double2* R) {
  __shared__ float tab[97 * kDrawThreads];
  const DrawSite ds(tab, tables, g.v3);
  if (!ds.live) return;
  const int site = ds.site;
  Stream st = streams[site];
  const SmemTable v = ds.view();
  for (int d = 0; d < 4; d++)
    for (int s = 0; s < g.ls; s++) {
      const float u1 = rano_dev(st, v);
      const float u2 = rano_dev(st, v);
      float a, b;
      box_muller(u1, u2, -1.0f, a, b);
      R[sidx(g, s, site, d)] = make_double2((double)a, (double)b);
    }
  streams[site] = st;
  ds.store(tables, g.v3);
}

// initialise_pp (evolution.F90:77-111): pp(:,:,:,mu) = sin part of gaussp, mu = 1..3
__global__ void __launch_bounds__(kDrawThreads) k_pp_draw(Stream* streams, float* tables, Geom g, float* pp) {
  __shared__ float tab[97 * kDrawThreads];
  const DrawSite ds(tab, tables, g.v3);
  if (!ds.live) return;
  const int site = ds.site;
  Stream st = streams[site];
  const SmemTable v = ds.view();
  for (int mu = 0; mu < 3; mu++) {
    const float u1 = rano_dev(st, v);
    const float u2 = rano_dev(st, v);
    float a, b;
    box_muller(u1, u2, -2.0f, a, b);
    pp[(size_t)mu * g.v3 + site] = a;
  }
  streams[site] = st;
  ds.store(tables, g.v3);
}

// one rano draw from the stream of `site`, written to *out
__global__ void k_rano_one(Stream* streams, float* tables, Geom g, int site, float* out) {
  Stream st = streams[site];
  *out = rano_dev(st, TableView{tables, g.v3, site});
  streams[site] = st;
}

inline unsigned site_grid(int v3) { return (unsigned)((v3 + 127) / 128); }
inline unsigned draw_grid(int v3) { return (unsigned)((v3 + kDrawThreads - 1) / kDrawThreads); }
}  // namespace

// ---------------------------------------------------------------- host side
int Rng::ensure(thr_ctx* c) {
  if (dev_streams) return THR_OK;
  if (cudaMalloc(&dev_streams, (size_t)c->g.v3 * sizeof(Stream)) != cudaSuccess) return THR_ERR_NOMEM;
  if (cudaMalloc(&dev_tables, (size_t)c->g.v3 * 97 * sizeof(float)) != cudaSuccess) return THR_ERR_NOMEM;
  return THR_OK;
}
void Rng::release() {
  cudaFree(dev_streams);
  cudaFree(dev_tables);
  dev_streams = nullptr;
  dev_tables = nullptr;
}

int rng_init(thr_ctx* c, double seed, int site_mode) {
  // G900ST needs an integer seed below 2^48 for its digit split to be exact
  if (!(seed >= 0.0) || seed >= 281474976710656.0 || seed != std::floor(seed)) return THR_ERR_BADARG;
  Rng& r = c->rng;
  r.site = site_mode != 0;
  r.ready = true;
  if (r.site) {
    THR_TRY(r.ensure(c));
    k_rng_init<<<site_grid(c->g.v3), 128, 0, c->st>>>((Stream*)r.dev_streams, (float*)r.dev_tables, c->g,
                                                       (uint64_t)seed);
    return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
  }
  // random.f90:119-126 with ip_global = 0
  r.hS = (uint64_t)seed;
  r.hidum = -1;
  Stream st{r.hS, r.hy, r.hidum};
  (void)rano_step(st, r.hv);
  r.hS = st.S;
  r.hy = st.y;
  r.hidum = st.idum;
  return THR_OK;
}

float rng_rano_host(Rng& r) {
  Stream st{r.hS, r.hy, r.hidum};
  float v = rano_step(st, r.hv);
  r.hS = st.S;
  r.hy = st.y;
  r.hidum = st.idum;
  return v;
}

// one gauss call into device ps[2][v3]
int rng_gauss_dev(thr_ctx* c, float scale, float* ps) {
  Rng& r = c->rng;
  if (!r.ready) return THR_ERR_BADARG;
  if (r.site) {
    k_gauss<<<draw_grid(c->g.v3), kDrawThreads, 0, c->st>>>((Stream*)r.dev_streams, (float*)r.dev_tables, c->g,
                                                             scale, ps);
    return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
  }
  // global stream: all first draws in Fortran site order, then all second draws (gaussian.F90:190-206)
  const int v3 = c->g.v3;
  std::vector<float> h(2 * (size_t)v3);
  std::vector<float> radius(v3);
  for (int i = 0; i < v3; i++) {
    const float lg = (float)std::log((double)rng_rano_host(r));
    radius[i] = sqrtf(scale * lg);
  }
  for (int i = 0; i < v3; i++) {
    const float th = kTpi * rng_rano_host(r);
    const float sn = (float)std::sin((double)th), cs = (float)std::cos((double)th);
    h[i] = radius[i] * sn;
    h[v3 + i] = radius[i] * cs;
  }
  // h is in natural (x fastest) order; scatter to storage order via the f3 converter (2 of 3 components)
  float* tmp = reinterpret_cast<float*>(c->stage);
  THR_CUDA(cudaMemcpyAsync(tmp, h.data(), 2 * (size_t)v3 * sizeof(float), cudaMemcpyHostToDevice, c->st));
  THR_CUDA(cudaStreamSynchronize(c->st));
  rng_natural_to_storage(c, ps, tmp, 2);
  return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
}

int rng_phi_draw(thr_ctx* c, double2* R) {
  Rng& r = c->rng;
  if (!r.ready) return THR_ERR_BADARG;
  if (r.site) {
    k_phi_draw<<<draw_grid(c->g.v3), kDrawThreads, 0, c->st>>>((Stream*)r.dev_streams, (float*)r.dev_tables, c->g,
                                                                R);
    return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
  }
  return THR_ERR_UNSUPPORTED;  // the global stream is drawn on the host by the caller
}

int rng_pp_draw(thr_ctx* c, float* pp) {
  Rng& r = c->rng;
  if (!r.ready) return THR_ERR_BADARG;
  if (r.site) {
    k_pp_draw<<<draw_grid(c->g.v3), kDrawThreads, 0, c->st>>>((Stream*)r.dev_streams, (float*)r.dev_tables, c->g,
                                                               pp);
    return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
  }
  return THR_ERR_UNSUPPORTED;
}

// one draw at 1-based site (ix, iy, it); result left in device *dout (site mode) or returned
int rng_rano_site(thr_ctx* c, int ix, int iy, int it, float* dout, float* hout) {
  Rng& r = c->rng;
  if (!r.ready) return THR_ERR_BADARG;
  if (!r.site) {
    float v = rng_rano_host(r);
    if (hout) *hout = v;
    if (dout) {
      r.hscratch = v;
      THR_CUDA(cudaMemcpyAsync(dout, &r.hscratch, sizeof(float), cudaMemcpyHostToDevice, c->st));
      THR_CUDA(cudaStreamSynchronize(c->st));
    }
    return THR_OK;
  }
  if (ix < 1 || iy < 1 || it < 1 || ix > c->g.lx || iy > c->g.ly || it > c->g.lt) return THR_ERR_BADARG;
  const int site = site_index(c->g, ix - 1, iy - 1, it - 1);
  float* target = dout;
  if (!target) target = reinterpret_cast<float*>(c->iscal + 512);
  k_rano_one<<<1, 1, 0, c->st>>>((Stream*)r.dev_streams, (float*)r.dev_tables, c->g, site, target);
  if (hout) {
    THR_CUDA(cudaMemcpyAsync(&r.hscratch, target, sizeof(float), cudaMemcpyDeviceToHost, c->st));
    THR_CUDA(cudaStreamSynchronize(c->st));
    *hout = r.hscratch;
  }
  return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
}

namespace {
__global__ void k_nat2sto(float* out, const float* in, Geom g, int ncomp) {
  int n = g.v3 * ncomp;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int r = i;
    int x = r % g.lx; r /= g.lx;
    int y = r % g.ly; r /= g.ly;
    int t = r % g.lt;
    int cc = r / g.lt;
    out[(size_t)cc * g.v3 + site_index(g, x, y, t)] = in[i];
  }
}
}  // namespace

void rng_natural_to_storage(thr_ctx* c, float* out, const float* in, int ncomp) {
  k_nat2sto<<<(unsigned)((c->g.v3 * ncomp + 255) / 256), 256, 0, c->st>>>(out, in, c->g, ncomp);
}

}  // namespace thr

using namespace thr;

extern "C" {

int thr_init_random(thr_ctx* c, double seed, int site_streams) {
  if (!c) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  THR_TRY(rng_init(c, seed, site_streams));
  return c->sync();
}

static int gauss_abi(thr_ctx* c, float* ps, float scale) {
  if (!c || !ps) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  void* buf;
  THR_TRY(c->buffer(thr_ctx::B_AUX, 2 * (size_t)c->g.v3 * sizeof(float), &buf));
  THR_TRY(rng_gauss_dev(c, scale, (float*)buf));
  to_fortran_ps(c->g, reinterpret_cast<float*>(c->stage), (const float*)buf, c->st);
  const size_t n = (size_t)(c->g.lx + 2) * (c->g.ly + 2) * (c->g.lt + 2) * 2;
  THR_CUDA(cudaMemcpyAsync(ps, c->stage, n * sizeof(float), cudaMemcpyDeviceToHost, c->st));
  return c->sync();
}

int thr_phi_draw_dev(thr_ctx* c, void* R) {
  if (!c || !R) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  return rng_phi_draw(c, (double2*)R);
}

int thr_gauss0(thr_ctx* c, float* ps) { return gauss_abi(c, ps, -1.0f); }
int thr_gaussp(thr_ctx* c, float* ps) { return gauss_abi(c, ps, -2.0f); }

int thr_rano(thr_ctx* c, int ix, int iy, int it, float* out) {
  if (!c || !out) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  return rng_rano_site(c, ix, iy, it, nullptr, out);
}

}  // extern "C"

// ---------------------------------------------------------------- generator state
namespace {
// host image of the whole random state: a header, then the streams and tables
struct RngImage {
  uint32_t magic, version;
  int32_t site, v3;
  uint64_t hS;
  float hy;
  int32_t hidum;
  float hv[97];
};
constexpr uint32_t kRngMagic = 0x54485252u;  // "RRHT"
}  // namespace

using namespace thr;

extern "C" {

int thr_rranget(thr_ctx* c, double* seed) {
  if (!c || !seed) return THR_ERR_BADARG;
  Rng& r = c->rng;
  if (!r.ready) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  if (!r.site) {
    *seed = (double)r.hS;
    return THR_OK;
  }
  Stream h;
  const int site = site_index(c->g, 0, 0, 0);  // rranget(seed, 1, 1, 1)
  THR_CUDA(cudaMemcpyAsync(&h, (const Stream*)r.dev_streams + site, sizeof(Stream), cudaMemcpyDeviceToHost, c->st));
  THR_CUDA(cudaStreamSynchronize(c->st));
  *seed = (double)h.S;
  return THR_OK;
}

int thr_rng_state_bytes(thr_ctx* c, unsigned long long* bytes) {
  if (!c || !bytes) return THR_ERR_BADARG;
  const size_t v3 = (size_t)c->g.v3;
  *bytes = sizeof(RngImage) + (c->rng.site ? v3 * (sizeof(Stream) + 97 * sizeof(float)) : 0);
  return THR_OK;
}

int thr_rng_save(thr_ctx* c, void* host) {
  if (!c || !host) return THR_ERR_BADARG;
  Rng& r = c->rng;
  if (!r.ready) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  RngImage im{};
  im.magic = kRngMagic;
  im.version = 1;
  im.site = r.site ? 1 : 0;
  im.v3 = c->g.v3;
  im.hS = r.hS;
  im.hy = r.hy;
  im.hidum = r.hidum;
  std::memcpy(im.hv, r.hv, sizeof(im.hv));
  std::memcpy(host, &im, sizeof(im));
  if (r.site) {
    char* p = (char*)host + sizeof(im);
    const size_t v3 = (size_t)c->g.v3;
    THR_CUDA(cudaMemcpyAsync(p, r.dev_streams, v3 * sizeof(Stream), cudaMemcpyDeviceToHost, c->st));
    THR_CUDA(cudaMemcpyAsync(p + v3 * sizeof(Stream), r.dev_tables, v3 * 97 * sizeof(float), cudaMemcpyDeviceToHost,
                             c->st));
    THR_CUDA(cudaStreamSynchronize(c->st));
  }
  return THR_OK;
}

int thr_rng_load(thr_ctx* c, const void* host) {
  if (!c || !host) return THR_ERR_BADARG;
  RngImage im;
  std::memcpy(&im, host, sizeof(im));
  if (im.magic != kRngMagic || im.version != 1) return THR_ERR_BADARG;
  if (im.site && im.v3 != c->g.v3) return THR_ERR_BADSHAPE;
  cudaSetDevice(c->dev);
  Rng& r = c->rng;
  r.site = im.site != 0;
  r.hS = im.hS;
  r.hy = im.hy;
  r.hidum = im.hidum;
  std::memcpy(r.hv, im.hv, sizeof(im.hv));
  if (r.site) {
    THR_TRY(r.ensure(c));
    const char* p = (const char*)host + sizeof(im);
    const size_t v3 = (size_t)c->g.v3;
    THR_CUDA(cudaMemcpyAsync(r.dev_streams, p, v3 * sizeof(Stream), cudaMemcpyHostToDevice, c->st));
    THR_CUDA(cudaMemcpyAsync(r.dev_tables, p + v3 * sizeof(Stream), v3 * 97 * sizeof(float), cudaMemcpyHostToDevice,
                             c->st));
    THR_CUDA(cudaStreamSynchronize(c->st));
  }
  r.ready = true;
  return THR_OK;
}

}  // extern "C"
