// thr_common.cuh -- shared device types for the B200 fermion hot path.
//
// Field layout in HBM (no halos; periodic neighbours are computed):
//   spinor  element (s, site, d) at  s + Ls*(site + V3*d)      (d = spin 0..3)
//           one contiguous plane per spin, the fifth dimension innermost, so a
//           warp reads 32 consecutive s of one spin plane in one transaction.
//   links   u[mu][site]  (mu = 0..2), antiperiodic t boundary already folded in
//           by coef (gauge.F90:30-32).
//   site    storage index of a 3D site; natural = x + Lx*(y + Ly*t), or the
//           even-odd order of lebesgue_eo.F90:49-51 (parity block, then
//           lexicographic inside the block).
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/thirring_b200.h"

namespace thr {

// ---------------------------------------------------------------- complex
template <class R> struct cplx;
template <> struct cplx<double> { using T = double2; };
template <> struct cplx<float> { using T = float2; };

__host__ __device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
__host__ __device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }

#define THR_CPLX_OPS(C, R)                                                                  \
  __host__ __device__ __forceinline__ C operator+(C a, C b) { return mk(a.x + b.x, a.y + b.y); } \
  __host__ __device__ __forceinline__ C operator-(C a, C b) { return mk(a.x - b.x, a.y - b.y); } \
  __host__ __device__ __forceinline__ C operator-(C a) { return mk(-a.x, -a.y); }                 \
  __host__ __device__ __forceinline__ C operator*(R s, C a) { return mk(s * a.x, s * a.y); }      \
  __host__ __device__ __forceinline__ C cmul(C a, C b) { return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); } \
  __host__ __device__ __forceinline__ C cconj(C a) { return mk(a.x, -a.y); }                      \
  /* conj(a)*b */                                                                              \
  __host__ __device__ __forceinline__ C cjmul(C a, C b) { return mk(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x); } \
  __host__ __device__ __forceinline__ C timesI(C a) { return mk(-a.y, a.x); }
THR_CPLX_OPS(double2, double)
THR_CPLX_OPS(float2, float)

// ---------------------------------------------------------------- storage
// Spinor storage types.  Arithmetic is FP64 for double2 storage and FP32 for
// the others (FP32 accumulation for BF16/FP16 storage).
template <class S> struct Sto;
template <> struct Sto<double2> {
  using R = double;
  using C = double2;
  static __device__ __forceinline__ C ld(const double2* p, size_t i) { return __ldg(p + i); }
  static __device__ __forceinline__ C ldcg(const double2* p, size_t i) { return __ldcg(p + i); }
  static __device__ __forceinline__ void st(double2* p, size_t i, C v) { p[i] = v; }
};
template <> struct Sto<float2> {
  using R = float;
  using C = float2;
  static __device__ __forceinline__ C ld(const float2* p, size_t i) { return __ldg(p + i); }
  static __device__ __forceinline__ C ldcg(const float2* p, size_t i) { return __ldcg(p + i); }
  static __device__ __forceinline__ void st(float2* p, size_t i, C v) { p[i] = v; }
};
template <> struct Sto<__nv_bfloat162> {
  using R = float;
  using C = float2;
  static __device__ __forceinline__ C ld(const __nv_bfloat162* p, size_t i) { return __bfloat1622float2(p[i]); }
  static __device__ __forceinline__ void st(__nv_bfloat162* p, size_t i, C v) { p[i] = __float22bfloat162_rn(v); }
};
template <> struct Sto<__half2> {
  using R = float;
  using C = float2;
  static __device__ __forceinline__ C ld(const __half2* p, size_t i) { return __half22float2(p[i]); }
  static __device__ __forceinline__ void st(__half2* p, size_t i, C v) { p[i] = __float22half2_rn(v); }
};

// ---------------------------------------------------------------- geometry
enum Layout { LAYOUT_NATURAL = 0, LAYOUT_EO = 1 };

struct Geom {
  int lx, ly, lt, ls;
  int v3;        // lx*ly*lt
  long long v5;  // ls*v3
  int layout;
  int hv3;       // v3/2 (even-odd)
  // division by a lattice extent d as a high multiply: q = umulhi(n, m) with
  // m = ceil(2^32 / d) equals n / d whenever n * d < 2^32 (the rounding excess
  // n * (m d - 2^32) / 2^32 < n d / 2^32 never reaches the next multiple);
  // 0 where a quotient range breaks that bound (plain division then)
  unsigned mdx = 0;  // for site / lx (natural) and k / (lx/2) (even-odd)
  unsigned mdy = 0;  // for row / ly
};

__host__ __device__ __forceinline__ unsigned geom_magic(long long nmax, int d) {
  if (d < 2 || (unsigned long long)nmax * (unsigned long long)d >= (1ULL << 32)) return 0u;
  return (unsigned)(((1ULL << 32) + (unsigned long long)d - 1) / (unsigned long long)d);
}

__host__ __device__ __forceinline__ Geom geom_make(int lx, int ly, int lt, int ls, int layout) {
  Geom g;
  g.lx = lx; g.ly = ly; g.lt = lt; g.ls = ls;
  g.v3 = lx * ly * lt;
  g.v5 = (long long)g.v3 * ls;
  g.layout = layout;
  g.hv3 = g.v3 / 2;
  g.mdx = layout == LAYOUT_EO ? geom_magic(g.hv3, lx >> 1) : geom_magic(g.v3, lx);
  g.mdy = geom_magic((long long)ly * lt, ly);
  return g;
}

// n / d for 0 <= n, with the magic multiplier m of d (0: divide)
__host__ __device__ __forceinline__ int geom_div(int n, int d, unsigned m) {
#ifdef __CUDA_ARCH__
  if (m) return (int)__umulhi((unsigned)n, m);
#else
  if (m) return (int)(((unsigned long long)(unsigned)n * m) >> 32);
#endif
  return n / d;
}

// 0-based coordinates of storage site `site`
__host__ __device__ __forceinline__ void site_coords(const Geom& g, int site, int& x, int& y, int& t) {
  if (g.layout == LAYOUT_EO) {
    int p = site >= g.hv3;
    int k = site - p * g.hv3;
    int hx = g.lx >> 1;
    int row = geom_div(k, hx, g.mdx);
    int xh = k - row * hx;
    t = geom_div(row, g.ly, g.mdy);
    y = row - t * g.ly;
    x = 2 * xh + ((p + y + t + 1) & 1);
  } else {
    int row = geom_div(site, g.lx, g.mdx);
    x = site - row * g.lx;
    t = geom_div(row, g.ly, g.mdy);
    y = row - t * g.ly;
  }
}

// storage site of 0-based coordinates (no wrapping)
__host__ __device__ __forceinline__ int site_index(const Geom& g, int x, int y, int t) {
  int n = x + g.lx * (y + g.ly * t);
  if (g.layout == LAYOUT_EO) {
    int p = (x + y + t + 1) & 1;  // mod(x+y+t, 2) with the reference's 1-based coordinates
    return p * g.hv3 + (n >> 1);
  }
  return n;
}

// forward / backward neighbour storage sites in direction mu (periodic)
struct Nbr {
  int f[3], b[3];
};
// `site` is the storage site of (x, y, t); in the natural order the neighbours
// are that index plus a stride, minus the extent at a periodic wrap
__host__ __device__ __forceinline__ Nbr neighbours(const Geom& g, int site, int x, int y, int t) {
  Nbr n;
  if (g.layout != LAYOUT_EO) {
    const int sy = g.lx, st = g.lx * g.ly;
    n.f[0] = site + (x + 1 == g.lx ? 1 - g.lx : 1);
    n.b[0] = site + (x == 0 ? g.lx - 1 : -1);
    n.f[1] = site + (y + 1 == g.ly ? sy - st : sy);
    n.b[1] = site + (y == 0 ? st - sy : -sy);
    n.f[2] = site + (t + 1 == g.lt ? st - g.v3 : st);
    n.b[2] = site + (t == 0 ? g.v3 - st : -st);
    return n;
  }
  int xp = x + 1 == g.lx ? 0 : x + 1, xm = x == 0 ? g.lx - 1 : x - 1;
  int yp = y + 1 == g.ly ? 0 : y + 1, ym = y == 0 ? g.ly - 1 : y - 1;
  int tp = t + 1 == g.lt ? 0 : t + 1, tm = t == 0 ? g.lt - 1 : t - 1;
  n.f[0] = site_index(g, xp, y, t);
  n.b[0] = site_index(g, xm, y, t);
  n.f[1] = site_index(g, x, yp, t);
  n.b[1] = site_index(g, x, ym, t);
  n.f[2] = site_index(g, x, y, tp);
  n.b[2] = site_index(g, x, y, tm);
  return n;
}

__host__ __device__ __forceinline__ size_t sidx(const Geom& g, int s, int site, int d) {
  return (size_t)s + (size_t)g.ls * ((size_t)site + (size_t)g.v3 * (size_t)d);
}
// the same in 32-bit arithmetic, for fields of fewer than 2^32 elements (checked
// by the stencil launchers): fewer instructions and registers in the hot loop
__host__ __device__ __forceinline__ unsigned sidx32(const Geom& g, int s, int site, int d) {
  return (unsigned)s + (unsigned)g.ls * ((unsigned)site + (unsigned)g.v3 * (unsigned)d);
}

// ---------------------------------------------------------------- gammas
// gammamatrices.F90:17-132 for mu = 1..3 (the hopping directions), values
// already multiplied by akappa = 1/2: gamma(mu,d) = 0.5 * (re + i*im) with
// re, im in {-1, 0, 1}; gin = target spin (0-based).
struct GammaEntry {
  signed char re, im, gin, pad;
};
__host__ __device__ constexpr GammaEntry gamma_entry(int mu, int d) {
  // mu=1: (-i,-i,i,i) -> (4,3,2,1); mu=2: (-1,1,1,-1) -> (4,3,2,1);
  // mu=3: (-i,i,i,-i) -> (3,4,1,2)
  return mu == 0 ? GammaEntry{0, (signed char)(d < 2 ? -1 : 1), (signed char)(3 - d), 0}
       : mu == 1 ? GammaEntry{(signed char)((d == 0 || d == 3) ? -1 : 1), 0, (signed char)(3 - d), 0}
                 : GammaEntry{0, (signed char)((d == 0 || d == 3) ? -1 : 1), (signed char)(d ^ 2), 0};
}

// gamma(mu,d) * z, exact (scaling by 1/2 and swaps only)
template <class C, class R>
__device__ __forceinline__ C gmul(GammaEntry e, C z) {
  const R h = R(0.5);
  if (e.re != 0) return (e.re > 0) ? mk(h * z.x, h * z.y) : mk(-(h * z.x), -(h * z.y));
  // +/- i * 0.5 * z
  return (e.im > 0) ? mk(-(h * z.y), h * z.x) : mk(h * z.y, -(h * z.x));
}

// (2 gamma(mu,d)) * z, exact: a sign and possibly a swap (2 gamma entries are +-1, +-i)
template <class C>
__device__ __forceinline__ C gp(GammaEntry e, C z) {
  if (e.re != 0) return e.re > 0 ? z : mk(-z.x, -z.y);
  return e.im > 0 ? mk(-z.y, z.x) : mk(z.y, -z.x);
}

// ---------------------------------------------------------------- dependent launch
// A kernel that the host launched as a programmatic dependent of the previous kernel on its
// stream may start before that kernel has finished: pdl_wait() blocks until it has finished
// and its writes are visible (a no-op for an ordinary launch), and pdl_trigger() lets this
// kernel's own dependent be launched now.  Every such kernel calls pdl_wait() before it
// touches memory its predecessor writes.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

}  // namespace thr
