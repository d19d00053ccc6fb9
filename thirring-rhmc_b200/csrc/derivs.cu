// derivs.cu -- fermion force dS/dtheta (derivs_module.F90:8-410).
//
// One warp owns one 3D site x: its lanes walk the fifth dimension (lane = s,
// coalesced loads of R and X2), accumulate the three link directions and
// combine them with a warp-shuffle reduction; lane 0 adds the result to
// dSdpi(x, mu).  No atomics: every output has exactly one owner.
//
// Shamir (derivs_shared, :99-196):
//   dSdpi(x,mu) += tk * sum_{s,d} Im[ conj R(s,x,d) X2(s,x+mu,d) - conj R(s,x+mu,d) X2(s,x,d) ]
//                + sg * tz * sum_{s,d} Im[ g(mu,d) ( conj R(s,x,d) X2(s,x+mu,g) + conj R(s,x+mu,d) X2(s,x,g) ) ]
//   tz = 2*real(anum) in single precision, tk = tz*akappa (single), sg = +1 (iflag 0) / -1.
// Wilson (derivs_wilson, :41-97) adds the slice terms of derivSlice (:348-410)
// for the neighbouring-slice pairs and the wall mass pairs (:198-249):
//   iflag 1: L = R(s) (all spins) with  X2(s+1)P-  [wall s=Ls: X2(1)P-,  c2]
//                                 and  X2(s-1)P+  [wall s=1:  X2(Ls)P+, c1]
//   iflag 0: L = P+R(s) with X2(s+1) [wall s=Ls: X2(1), c2]
//            L = P-R(s) with X2(s-1) [wall s=1:  X2(Ls), c1]
//   c1 = -am | -i am, c2 = -am | +i am (imass 1 | 3), dmult = -1 for iflag 1.
#include "ctx.h"
#include "derivs.h"

namespace thr {

namespace {

// Im(c * conj(a) * b)
__device__ __forceinline__ double im_cjab(double2 c, double2 a, double2 b) {
  double2 t = cjmul(a, b);  // conj(a) b
  return c.x * t.y + c.y * t.x;
}
__device__ __forceinline__ double2 gmul_d(GammaEntry e, double2 z) { return gmul<double2, double>(e, z); }

// KER 0 (Shamir) / 1 (Wilson, adds the slice terms); MINB resident 256-thread blocks per SM
// bound the registers.  The site's own spinors R(x), X2(x) are loaded once and serve all
// three directions; per direction only the forward neighbour's are loaded.
template <int KER, int MINB>
__global__ void __launch_bounds__(256, MINB) k_derivs(double* __restrict__ dS, const double2* __restrict__ R,
                                                      const double2* __restrict__ X2, Geom g, int iflag, double tk,
                                                      double tz, double2 c1, double2 c2) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= g.v3) return;
  const int site = warp;
  int x, y, t;
  site_coords(g, site, x, y, t);
  const Nbr nb = neighbours(g, site, x, y, t);
  const double sg = (iflag == 0) ? 1.0 : -1.0;
  double accm[3] = {0.0, 0.0, 0.0};
  const int Ls = g.ls;
  for (int s = lane; s < Ls; s += 32) {
    double2 Rx[4], Xx[4];
#pragma unroll
    for (int d = 0; d < 4; d++) {
      Rx[d] = __ldg(R + sidx(g, s, site, d));
      Xx[d] = __ldg(X2 + sidx(g, s, site, d));
    }
#pragma unroll
    for (int mu = 0; mu < 3; mu++) {
      const int xf = nb.f[mu];
      double2 Rf[4], Xf[4];
#pragma unroll
      for (int d = 0; d < 4; d++) {
        Rf[d] = __ldg(R + sidx(g, s, xf, d));
        Xf[d] = __ldg(X2 + sidx(g, s, xf, d));
      }
      double a1 = 0.0, a2 = 0.0;
#pragma unroll
      for (int d = 0; d < 4; d++) {
        const GammaEntry ge = gamma_entry(mu, d);
        const int gi = ge.gin;
        double2 t1 = cjmul(Rx[d], Xf[d]), t2 = cjmul(Rf[d], Xx[d]);
        a1 += t1.y - t2.y;
        double2 t3 = cjmul(Rx[d], Xf[gi]) + cjmul(Rf[d], Xx[gi]);
        a2 += gmul_d(ge, t3).y;
      }
      double acc = tk * a1 + sg * tz * a2;
      if (KER == 1) {
        // slice terms: partner slice in X2 at s+1 (P-, wall c2) and s-1 (P+, wall c1)
#pragma unroll
        for (int side = 0; side < 2; side++) {
          const bool up = side == 0;  // partner s+1 (P- for iflag 1)
          const int sp = up ? (s < Ls - 1 ? s + 1 : 0) : (s > 0 ? s - 1 : Ls - 1);
          const bool wall = up ? (s == Ls - 1) : (s == 0);
          const double2 cm = wall ? (up ? c2 : c1) : make_double2(1.0, 0.0);
          double2 Px[4], Pf[4];
#pragma unroll
          for (int d = 0; d < 4; d++) {
            Px[d] = __ldg(X2 + sidx(g, sp, site, d));
            Pf[d] = __ldg(X2 + sidx(g, sp, xf, d));
          }
          double b1 = 0.0, b2 = 0.0;
#pragma unroll
          for (int d = 0; d < 4; d++) {
            const GammaEntry ge = gamma_entry(mu, d);
            const int gi = ge.gin;
            bool kd, kg;
            if (iflag == 1) {  // L all spins, partner masked: P- (2,3) up, P+ (0,1) down
              kd = up ? (d >= 2) : (d < 2);
              kg = up ? (gi >= 2) : (gi < 2);
            } else {  // L masked: P+ (0,1) pairs up, P- (2,3) pairs down; partner all spins
              kd = kg = up ? (d < 2) : (d >= 2);
            }
            if (kd) b1 += im_cjab(cm, Rx[d], Pf[d]) - im_cjab(cm, Rf[d], Px[d]);
            if (kg) {
              const double2 cgm = cmul(cm, gmul_d(ge, make_double2(1.0, 0.0)));
              b2 += im_cjab(cgm, Rx[d], Pf[gi]) + im_cjab(cgm, Rf[d], Px[gi]);
            }
          }
          acc += tk * b1 + sg * tz * b2;
        }
      }
      accm[mu] += acc;
    }
  }
#pragma unroll
  for (int mu = 0; mu < 3; mu++) {
    double v = accm[mu];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) dS[(size_t)mu * g.v3 + site] += v;
  }
}

}  // namespace

int launch_derivs(thr_ctx* c, double* dS, const double2* R, const double2* X2, double anum, int iflag, float am,
                  int imass) {
  if (iflag != 0 && iflag != 1) return THR_ERR_BADARG;
  if (c->p.kernel == 1 && imass != 1 && imass != 3) return THR_ERR_UNSUPPORTED;
  const float tzf = 2.0f * (float)anum;  // tzi_real = 2*real(anum): derivs_module.F90:126
  const double tz = (double)tzf;
  const double tk = (double)(tzf * 0.5f);  // tzi_real*real(akappa)
  const double a = (double)am;
  const double2 c1 = imass == 1 ? make_double2(-a, 0.0) : make_double2(0.0, -a);
  const double2 c2 = imass == 1 ? make_double2(-a, 0.0) : make_double2(0.0, a);
  const int threads = 256;
  const unsigned blocks = (unsigned)(((size_t)c->g.v3 * 32 + threads - 1) / threads);
  if (c->p.kernel == 1)
    k_derivs<1, 1><<<blocks, threads, 0, c->st>>>(dS, R, X2, c->g, iflag, tk, tz, c1, c2);
  else
    k_derivs<0, 3><<<blocks, threads, 0, c->st>>>(dS, R, X2, c->g, iflag, tk, tz, c1, c2);
  return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
}

}  // namespace thr
