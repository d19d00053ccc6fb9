// dslash.cu -- domain-wall Dirac operator M and M^dagger on one B200.
//
// One thread owns one 5D site (s, x, y, t) and all four spin components.
// A block is (Ls lanes) x (sites per block); consecutive threads read
// consecutive s of one spin plane, so every load is a coalesced 512-byte
// warp transaction (FP64).  The six spatial neighbours are periodic index
// arithmetic: the halo exchange of comms5.F90 is folded into the indexing,
// and the antiperiodic time boundary lives in the links (gauge.F90:30-32).
//
// Shamir kernel: dirac.F90:29-179 (M) and :303-494 (M^dagger), one pass.
// Wilson kernel: dirac.F90:226-301 (M) and :539-626 (M^dagger).  The
// reference applies the 3D Wilson operator D_W to 2*Ls+2 projected slices;
// by linearity of D_W each output slice is
//   M:      Phi(s) = D_W Q(s) + 2 R(s) - Q(s),
//           Q(s) = R(s) + P+ R(s-1) + P- R(s+1)   (walls: c1 P+ R(Ls), c2 P- R(1))
//   M^dag:  Phi(s)[P-] = D_W^dag Qm(s) + 2 R(s) - Qm(s),  Qm = R(s) + R(s-1) (wall z R(Ls))
//           Phi(s)[P+] = D_W^dag Qp(s) + 2 R(s) - Qp(s),  Qp = R(s) + R(s+1) (wall z' R(1))
// so the whole operator is again one pass over memory.
//
// The per-site arithmetic lives in shamir_site / wilson_site; the single-
// lattice kernels and the batched kernel (many right-hand sides or many
// lattices of different shapes in one persistent launch) share it.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>

#include "batch.h"
#include "ctx.h"
#include "dslash_site.cuh"
#include "thr_common.cuh"
#include "thr_kernels.h"

namespace thr {

// one FP64 partial per block, fixed reduction order
__device__ __forceinline__ void block_partial(double v, double* out) {
  __shared__ double sh[32];
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int nthr = blockDim.x * blockDim.y;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((tid & 31) == 0) sh[tid >> 5] = v;
  __syncthreads();
  if (tid < 32) {
    const int nw = (nthr + 31) >> 5;
    v = tid < nw ? sh[tid] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (tid == 0) *out = v;
  }
  __syncthreads();
}

// ---------------------------------------------------------------- overlap
// The Zolotarev domain-wall operator of measure_OWilson.F90 (odslash :14-89,
// odslashd :91-167): the Wilson-kernel operator with slice s's 3D Wilson term
// D_W = DWilson(-am3) scaled by its coefficient c[s] (prepZolo, :169-188) and
// the imass 3 walls of the opposite sign.  By linearity
//   M:      Phi(s) = c[s] D_W Q(s) + 2 R(s) - Q(s),
//           Q(s) = R(s) + P- R(s+1) + P+ R(s-1)   (walls: m1 P+ R(Ls) into s = 1,
//           m2 P- R(1) into s = Ls; m1 = -am | +i am, m2 = -am | -i am)
//   M^dag:  Phi(s)[P+] = D_W^dag(c[s] R(s) + c[s+1] R(s+1)) + R(s) - R(s+1)
//           (s = Ls: c[Ls] R(Ls) + z2 c[1] R(1), non-D part R(Ls) - z2 R(1), z2 = -am | -i am)
//           Phi(s)[P-] = D_W^dag(c[s] R(s) + c[s-1] R(s-1)) + R(s) - R(s-1)
//           (s = 1: c[1] R(1) + z1 c[Ls] R(Ls), non-D part R(1) - z1 R(Ls), z1 = -am | +i am)
// (1-based slices as in the reference).  One thread per 5D site, FP64.
template <bool DAG>
__device__ __forceinline__ void overlap_site(const double2* __restrict__ in, const double2* __restrict__ u,
                                             const Geom& g, int s, int site, float am, int imass, float am3,
                                             const double* __restrict__ zc, double2* res) {
  using C = double2;
  using R = double;
  int x, y, t;
  site_coords(g, site, x, y, t);
  const Nbr nb = neighbours(g, site, x, y, t);
  SpinorView<double2> Rv{in, g};
  const int Ls = g.ls;
  const R a = (R)am;
  const R dgw = (R)(3.0f + (-am3));  // DWilson(..., -am3) diagonal: dirac.F90:191, :505
  const R cs = __ldg(zc + s);
  if (!DAG) {
    const C m1 = imass == 1 ? mk(-a, R(0)) : mk(R(0), a);   // measure_OWilson.F90:66-71
    const C m2 = imass == 1 ? mk(-a, R(0)) : mk(R(0), -a);  // :78-83
    C q[4];
    wilson_q<double2>(Rv, s, site, Ls, m1, m2, q);
#pragma unroll
    for (int d = 0; d < 4; d++) res[d] = (cs * dgw - R(1)) * q[d] + R(2) * Rv(s, site, d);
#pragma unroll
    for (int mu = 0; mu < 3; mu++) {
      const C U = cs * __ldg(u + (size_t)mu * g.v3 + site);
      const C Ub = cs * cconj(__ldg(u + (size_t)mu * g.v3 + nb.b[mu]));
      wilson_q<double2>(Rv, s, nb.f[mu], Ls, m1, m2, q);
      hop_projected<C, R>(mu, true, U, q, res);
      wilson_q<double2>(Rv, s, nb.b[mu], Ls, m1, m2, q);
      hop_projected<C, R>(mu, false, Ub, q, res);
    }
  } else {
    const C z1 = imass == 1 ? mk(-a, R(0)) : mk(R(0), a);   // upper right, measure_OWilson.F90:139-144
    const C z2 = imass == 1 ? mk(-a, R(0)) : mk(R(0), -a);  // lower left, :152-157
    // output spins 0,1 from slice s+1 (wall: slice 0 with z2), spins 2,3 from s-1 (wall: Ls-1, z1);
    // one pass over the neighbours loads R(s) and both partner slices once
    const bool in0 = s < Ls - 1, in1 = s > 0;
    const int sp0 = in0 ? s + 1 : 0, sp1 = in1 ? s - 1 : Ls - 1;
    const R cn0 = __ldg(zc + sp0), cn1 = __ldg(zc + sp1);
    const C zb0 = cn0 * z2, zb1 = cn1 * z1;
    auto qpair = [&](int st, C* q0, C* q1) {
#pragma unroll
      for (int d = 0; d < 4; d++) {
        const C r = Rv(s, st, d), a0 = Rv(sp0, st, d), a1 = Rv(sp1, st, d);
        q0[d] = in0 ? cs * r + cn0 * a0 : cs * r + cmul(zb0, a0);
        q1[d] = in1 ? cs * r + cn1 * a1 : cs * r + cmul(zb1, a1);
      }
    };
    {
      C q0[4], q1[4];
      qpair(site, q0, q1);
#pragma unroll
      for (int d = 0; d < 4; d++) {
        const bool lo = d < 2;
        const C a2 = Rv(lo ? sp0 : sp1, site, d);
        const C xo = (lo ? in0 : in1) ? a2 : cmul(lo ? z2 : z1, a2);
        res[d] = dgw * (lo ? q0[d] : q1[d]) + Rv(s, site, d) - xo;
      }
    }
#pragma unroll
    for (int mu = 0; mu < 3; mu++) {
      const C U = __ldg(u + (size_t)mu * g.v3 + site);
      const C Ub = cconj(__ldg(u + (size_t)mu * g.v3 + nb.b[mu]));
#pragma unroll
      for (int dir = 0; dir < 2; dir++) {
        C q0[4], q1[4];
        qpair(dir == 0 ? nb.f[mu] : nb.b[mu], q0, q1);
        const C W = dir == 0 ? U : Ub;
#pragma unroll
        for (int d = 0; d < 4; d++) {
          const C* q = d < 2 ? q0 : q1;
          const GammaEntry ge = gamma_entry(mu, d);
          const C gq = gp(ge, q[ge.gin]);
          res[d] = res[d] - R(0.5) * cmul(W, dir == 0 ? q[d] + gq : q[d] - gq);
        }
      }
    }
  }
}

// odslash / odslashd on one lattice: blockDim = (Ls, sites per block) as the Wilson kernel's
template <bool DAG, int MINB>
__global__ void __launch_bounds__(256, MINB)
    k_odslash(double2* __restrict__ out, const double2* __restrict__ in, const double2* __restrict__ u, Geom g,
              float am, int imass, float am3, const double* __restrict__ zc, const int* skip) {
  if (skip && *skip) return;
  const int s = threadIdx.x;
  const int site = blockIdx.x * blockDim.y + threadIdx.y;
  if (site >= g.v3) return;
  double2 acc[4];
  overlap_site<DAG>(in, u, g, s, site, am, imass, am3, zc, acc);
#pragma unroll
  for (int d = 0; d < 4; d++) Sto<double2>::st(out, sidx32(g, s, site, d), acc[d]);
}

// ---------------------------------------------------------------- kernels
// One thread per 5D site: blockDim = (Ls, sites per block), NT threads at most.
// Shamir blocks are small (NT = 128, 8 resident per SM at <= 64 registers):
// the kernel is latency-bound, and small blocks keep more loads in flight.
// MINB (resident blocks per SM the register budget is cut for) is chosen per
// lattice by the autotuner below; it changes register allocation only, so the
// results are bit-identical whichever value runs.
//
// Epilogues (EPI): 0 store out = M in; 2 also one FP64 partial per block of
// |out|^2; 1 the residual update of the multishift solver fused in -- out =
// aux + (*coef) * (M in), with M in never stored, and a partial of |out|^2;
// 3 out = M in + (*coef) * aux with a partial of |out|^2 (the batched
// multishift keeps h = M p by this recurrence instead of storing p).
template <class S, int KER, bool DAG, int EPI, int NT, bool SHFL, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    k_dslash(S* __restrict__ out, const S* __restrict__ in, const typename Sto<S>::C* __restrict__ u, Geom g, float am,
             int imass, float am3, const int* skip, const S* __restrict__ aux, const double* __restrict__ coef,
             double* __restrict__ partials, int rev) {
  pdl_wait();
  pdl_trigger();
  if (skip && *skip) return;
  using R = typename Sto<S>::R;
  const R om = (EPI == 1 || EPI == 3) ? (R)(*coef) : R(0);
  // rev: blocks walk the sites from the top, so that the first blocks find the
  // end of a field the previous kernel has just written still in L2
  const int bid = rev ? (int)gridDim.x - 1 - (int)blockIdx.x : (int)blockIdx.x;
  dslash_block<S, KER, DAG, EPI, NT, SHFL>(out, in, u, g, am, imass, am3, aux, om, bid, partials);
}

// Shamir kernel with K site groups per block (sites per CTA): blockDim = (Ls, K x the
// sites of a k_dslash block), where a k_dslash block (Ls x sites threads) is whole warps
// (128 threads for Ls 32, 16, 8; 96 for Ls 48).  Each group computes as one k_dslash
// block and writes that block's partial (partials[K bid + group], the same grouping,
// order and index), so the results are the same bits; the autotuner times it as
// candidates kG2Code + 10 K + MINB.
template <class S, bool DAG, int EPI, bool SHFL, int K, int MINB>
__global__ void __launch_bounds__(128 * K, MINB)
    k_dslash_g2(S* __restrict__ out, const S* __restrict__ in, const typename Sto<S>::C* __restrict__ u, Geom g,
                float am, int imass, float am3, const int* skip, const S* __restrict__ aux,
                const double* __restrict__ coef, double* __restrict__ partials, int rev, int np) {
  pdl_wait();
  pdl_trigger();
  if (skip && *skip) return;
  using C = typename Sto<S>::C;
  using R = typename Sto<S>::R;
  const R om = (EPI == 1 || EPI == 3) ? (R)(*coef) : R(0);
  const int bid = rev ? (int)gridDim.x - 1 - (int)blockIdx.x : (int)blockIdx.x;
  const int s = threadIdx.x;
  double racc = 0.0;
  const int site = bid * (int)blockDim.y + threadIdx.y;
  const bool live = site < g.v3;
  if (SHFL || live) {  // with SHFL every lane takes part (spare rows on a clamped site)
    const int st = live ? site : g.v3 - 1;
    C acc[4];
    apply_site<S, 0, DAG, SHFL>(in, u, g, s, st, am, imass, am3, acc);
    if (live) {
#pragma unroll
      for (int d = 0; d < 4; d++) epi_element<S, EPI, false>(out, aux, om, sidx32(g, s, site, d), acc[d], racc);
    }
  }
  if (EPI != 0) {
    __shared__ double red[128 * K];
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int gsz = (int)(blockDim.x * blockDim.y) / K;  // threads of one group (whole warps)
    red[tid] = racc;
    __syncthreads();
    const int grp = tid / gsz, lt = tid - grp * gsz;
    if (lt < 32) {
      double v = 0.0;
      for (int i = lt; i < gsz; i += 32) v += red[grp * gsz + i];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lt == 0 && K * bid + grp < np) partials[K * bid + grp] = v;
    }
  }
}

// Shamir kernel with four threads per 5D site, for lattices too small to fill the GPU
// with one thread per site (at 12^2x12, Ls 16 the one-thread kernel has 1.5 warps per
// scheduler, and each warp's ~570 dependent instructions set the launch's latency).
// blockDim = (Ls, sites per block, 4) over the sites of a 128-thread k_dslash block:
// threadIdx.z = 0 owns the site (the local terms of shamir_local, then the six hops'
// contributions in shamir_site's order, the epilogue and the block's partial), z = 1..3
// form the products W h(d) of the forward and backward hop in direction z - 1
// (hop_products) and hand them over in shared memory.  Each output element gets the
// same operations in the same order as in k_dslash, and the partials group the same
// sites, so the results are the same bits; it is one more register-budget candidate of
// the autotuner (code kSplitCode), which keeps it only where it is faster.
// the products of one helper thread: direction MU (a compile-time constant, so that the
// spin permutation indexes registers), forward and backward hop
template <class S, bool DAG, int MU>
__device__ __forceinline__ void split_products(const S* __restrict__ in, const typename Sto<S>::C* __restrict__ u,
                                               const Geom& g, int s, int site, typename Sto<S>::C (*wh_s)[2][2][128],
                                               int slot) {
  using C = typename Sto<S>::C;
  int x, y, t;
  site_coords(g, site, x, y, t);
  const Nbr nb = neighbours(g, site, x, y, t);
  SpinorView<S> Rv{in, g};
#pragma unroll
  for (int dir = 0; dir < 2; dir++) {
    const int ns = dir == 0 ? nb.f[MU] : nb.b[MU];
    const C W = dir == 0 ? __ldg(u + (size_t)MU * g.v3 + site) : cconj(__ldg(u + (size_t)MU * g.v3 + nb.b[MU]));
    C r[4];
#pragma unroll
    for (int d = 0; d < 4; d++) r[d] = Rv(s, ns, d);
    C wh[2];
    hop_products<C>(MU, (dir == 0) != DAG, W, r, wh);
    wh_s[MU][dir][0][slot] = wh[0];
    wh_s[MU][dir][1][slot] = wh[1];
  }
}

template <class S, bool DAG, int EPI, bool SHFL>
__global__ void __launch_bounds__(512, 2)
    k_dslash_split(S* __restrict__ out, const S* __restrict__ in, const typename Sto<S>::C* __restrict__ u, Geom g,
                   float am, int imass, float am3, const int* skip, const S* __restrict__ aux,
                   const double* __restrict__ coef, double* __restrict__ partials, int rev) {
  pdl_wait();
  pdl_trigger();
  if (skip && *skip) return;
  using C = typename Sto<S>::C;
  using R = typename Sto<S>::R;
  __shared__ C wh_s[3][2][2][128];  // [mu][dir][d][s + Ls * site in block]
  const int s = threadIdx.x, zi = threadIdx.y, role = threadIdx.z;
  const int slot = s + (int)blockDim.x * zi;
  const int bid = rev ? (int)gridDim.x - 1 - (int)blockIdx.x : (int)blockIdx.x;
  const int site = bid * (int)blockDim.y + zi;
  const bool live = site < g.v3;
  C acc[4];
  if (role > 0) {
    if (live) {
      if (role == 1) split_products<S, DAG, 0>(in, u, g, s, site, wh_s, slot);
      else if (role == 2) split_products<S, DAG, 1>(in, u, g, s, site, wh_s, slot);
      else split_products<S, DAG, 2>(in, u, g, s, site, wh_s, slot);
    }
  } else if (SHFL || live) {  // with SHFL every owner lane takes part (spare rows on a clamped site)
    shamir_local<S, DAG, SHFL>(in, g, s, live ? site : g.v3 - 1, am, imass, am3, acc);
  }
  __syncthreads();
  double racc = 0.0;
  if (role == 0 && live) {
#pragma unroll
    for (int mu = 0; mu < 3; mu++) {
#pragma unroll
      for (int dir = 0; dir < 2; dir++) {
        const C wh[2] = {wh_s[mu][dir][0][slot], wh_s[mu][dir][1][slot]};
        hop_accumulate<C, R>(mu, (dir == 0) != DAG, wh, acc);
      }
    }
    const R om = (EPI == 1 || EPI == 3) ? (R)(*coef) : R(0);
#pragma unroll
    for (int d = 0; d < 4; d++) epi_element<S, EPI, false>(out, aux, om, sidx32(g, s, site, d), acc[d], racc);
  }
  if (EPI != 0) {
    // the partial of k_dslash's block: the owners' values in slot order, summed by the
    // first warp (all owners: the owners are the block's first Ls x sites threads)
    __shared__ double red[128];
    const int nown = (int)(blockDim.x * blockDim.y);
    if (role == 0) red[slot] = racc;
    __syncthreads();
    if (role == 0 && slot < 32) {
      double v = 0.0;
      for (int i = slot; i < nown; i += 32) v += red[i];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (slot == 0) partials[bid] = v;
    }
  }
}

// Shamir kernel, even Ls, FP32 storage: one thread owns two consecutive s of a
// site (s0 = 2 threadIdx.x and s0 + 1), so every spinor access is one 16-byte
// load or store (float4) instead of two 8-byte ones; the arithmetic per element
// is that of shamir_site.  blockDim = (Ls / 2, sites per block) with the sites
// per block of the one-s kernel, so the grid -- and the partials of the
// epilogues -- are the same; blocks have about 64 threads, 16 per SM.  (Written
// for either complex type; for FP64 storage it ran at 45-49 us against the
// one-s kernel's 38 us on the 32^2x32, Ls 32 lattice, so FP64 keeps one s per
// thread.)
__device__ __forceinline__ void ld_pair(const float2* p, unsigned i, float2& a, float2& b) {
  const float4 v = __ldg(reinterpret_cast<const float4*>(p + i));
  a = make_float2(v.x, v.y);
  b = make_float2(v.z, v.w);
}
__device__ __forceinline__ void ld_pair(const double2* p, unsigned i, double2& a, double2& b) {
  a = __ldg(p + i);
  b = __ldg(p + i + 1);
}
__device__ __forceinline__ void st_pair(float2* p, unsigned i, float2 a, float2 b) {
  *reinterpret_cast<float4*>(p + i) = make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ void st_pair(double2* p, unsigned i, double2 a, double2 b) {
  p[i] = a;
  p[i + 1] = b;
}
template <class C, bool DAG, int EPI, int MINB>
__global__ void __launch_bounds__(64, MINB)
    k_dslash_pair(C* __restrict__ out, const C* __restrict__ in, const C* __restrict__ u, Geom g, float am,
                  int imass, float am3, const int* skip, const C* __restrict__ aux, const double* __restrict__ coef,
                  double* __restrict__ partials, int rev) {
  pdl_wait();
  pdl_trigger();
  if (skip && *skip) return;
  using R = typename Sto<C>::R;
  const R om = (EPI == 1 || EPI == 3) ? (R)(*coef) : R(0);
  const int s0 = 2 * threadIdx.x;
  const int bid = rev ? (int)gridDim.x - 1 - (int)blockIdx.x : (int)blockIdx.x;
  const int site0 = bid * blockDim.y + threadIdx.y;
  const bool live = site0 < g.v3;
  double racc = 0.0;
  if (live) {
    const int site = site0;
    int x, y, t;
    site_coords(g, site, x, y, t);
    const Nbr nb = neighbours(g, site, x, y, t);
    SpinorView<C> Rv{in, g};
    const int Ls = g.ls;
    const R diag = (R)((3.0f - am3) + 1.0f);
    C c0[4], c1[4], a0c[4], a1c[4];
#pragma unroll
    for (int d = 0; d < 4; d++) {
      ld_pair(in, sidx32(g, s0, site, d), c0[d], c1[d]);
      a0c[d] = diag * c0[d];
      a1c[d] = diag * c1[d];
    }
    const int A = DAG ? 0 : 2, B = DAG ? 2 : 0;  // spins taking R(s+1) / R(s-1)
#pragma unroll
    for (int k = 0; k < 2; k++) {
      a0c[A + k] = a0c[A + k] - c1[A + k];                                   // s0 + 1 = s1 < Ls
      if (s0 + 1 < Ls - 1) a1c[A + k] = a1c[A + k] - Rv(s0 + 2, site, A + k);
      if (s0 > 0) a0c[B + k] = a0c[B + k] - Rv(s0 - 1, site, B + k);
      a1c[B + k] = a1c[B + k] - c0[B + k];                                   // s1 - 1 = s0
    }
    const R a = (R)am;
    const bool five = imass == 5;
    const C cA = imass == 1 ? mk(a, R(0)) : mk(R(0), (five && DAG) ? -a : a);
    const C cB = imass == 1 ? mk(a, R(0)) : mk(R(0), five ? (DAG ? -a : a) : -a);
#pragma unroll
    for (int k = 0; k < 2; k++) {
      if (s0 + 1 == Ls - 1) a1c[A + k] = a1c[A + k] + cmul(cA, five ? c1[B + k] : Rv(0, site, A + k));
      if (s0 == 0) a0c[B + k] = a0c[B + k] + cmul(cB, five ? c0[A + k] : Rv(Ls - 1, site, B + k));
    }
#pragma unroll
    for (int mu = 0; mu < 3; mu++) {
#pragma unroll
      for (int dir = 0; dir < 2; dir++) {
        const int ns = dir == 0 ? nb.f[mu] : nb.b[mu];
        const C W = dir == 0 ? __ldg(u + (size_t)mu * g.v3 + site) : cconj(__ldg(u + (size_t)mu * g.v3 + nb.b[mu]));
        C r0[4], r1[4];
#pragma unroll
        for (int d = 0; d < 4; d++) ld_pair(in, sidx32(g, s0, ns, d), r0[d], r1[d]);
        hop_projected<C, R>(mu, (dir == 0) != DAG, W, r0, a0c);
        hop_projected<C, R>(mu, (dir == 0) != DAG, W, r1, a1c);
      }
    }
#pragma unroll
    for (int d = 0; d < 4; d++) {
      const unsigned i = sidx32(g, s0, site, d);
      C v0 = a0c[d], v1 = a1c[d];
      if (EPI == 1) {
        C q0, q1;
        ld_pair(aux, i, q0, q1);
        v0 = q0 + om * v0;  // r = r + omega*s (multishift_module.F90:137)
        v1 = q1 + om * v1;
      } else if (EPI == 3) {
        C q0, q1;
        ld_pair(aux, i, q0, q1);
        v0 = v0 + om * q0;  // h = M r + gamma h
        v1 = v1 + om * q1;
      }
      st_pair(out, i, v0, v1);
      if (EPI != 0) racc += epi_norm<C>(v0) + epi_norm<C>(v1);
    }
  }
  if (EPI != 0) {
    __shared__ double red[64];
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int nthr = blockDim.x * blockDim.y;
    red[tid] = racc;
    __syncthreads();
    if (tid < 32) {
      double v = 0.0;
      for (int i = tid; i < nthr; i += 32) v += red[i];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (tid == 0) partials[bid] = v;
    }
  }
}

// ---------------------------------------------------------------- Shamir, staged tiles
// FP64 Shamir kernel for the natural site order with Lx, Ly divisible by 4, Lt
// by 2 and Ls by 8.  A block owns a 4x4x2 tile of sites and 8 consecutive s
// (256 threads: s fastest, then x, y, t).  One thread first stages everything
// the block's sites read into shared memory with 11 TMA tensor copies (no
// multicast) completing on one mbarrier: the tile's spinors with one s on
// either side (the s-neighbours), the six one-site faces around the tile, and
// the links of the tile and of its three lower faces.  The spinor field is a
// 5D tensor (2 Ls doubles, Lx, Ly, Lt, 4 spins), the links one of (2 doubles,
// Lx, Ly, Lt, 3); a box of the tile or of a face lands in shared memory in
// that dimension order.  At the ends of the fifth dimension the s-neighbour
// slots lie outside the tensor (filled with zeros) and take the wall values
// R(Ls-1) and R(0) instead, loaded by the block's threads while the copies are
// in flight.  The arithmetic is then shamir_site's, operation for operation,
// with every operand from shared memory: a 5D site costs 3.4 spinor reads from
// L2 (tile plus faces) instead of 7, and neither load latency nor address
// arithmetic sits inside it.  54 KB of shared memory per block, 4 blocks
// (1024 threads) per SM.
namespace tile {
constexpr int TX = 4, TY = 4, TT = 2, SC = 8;
constexpr int NT = TX * TY * TT * SC;  // 256 threads
constexpr int NS = TX * TY * TT;       // 32 sites
constexpr int CW = SC + 2;             // centre row: s0 - 1 .. s0 + SC
// regions of the shared tile (offsets in double2, each a multiple of 8 = 128 bytes)
constexpr int CEN = 0;                        // [d][t][y][x][CW]
constexpr int XFD = TT * TY * SC;             // x faces [dir][d][t][y][SC]: spin stride
constexpr int YFD = TT * TX * SC;             // y faces [dir][d][t][x][SC]
constexpr int TFD = TY * TX * SC;             // t faces [dir][d][y][x][SC]
constexpr int XF = CEN + 4 * NS * CW;
constexpr int YF = XF + 2 * 4 * XFD;
constexpr int TF = YF + 2 * 4 * YFD;
constexpr int UT = TF + 2 * 4 * TFD;          // [mu][t][y][x]  links of the tile
constexpr int UX = UT + 3 * NS;               // [t][y]  u(0) on the x - 1 face
constexpr int UY = UX + TT * TY;              // [t][x]  u(1) on the y - 1 face
constexpr int UTM = UY + TT * TX;             // [y][x]  u(2) on the t - 1 face
constexpr int END = UTM + TY * TX;            // 3456 double2 = 54 KB
constexpr int SMEM = END * (int)sizeof(double2) + 128;  // + alignment slack
static_assert(XF % 8 == 0 && YF % 8 == 0 && TF % 8 == 0 && UT % 8 == 0 && UX % 8 == 0 && UY % 8 == 0 &&
                  UTM % 8 == 0 && (4 * XFD) % 8 == 0 && (4 * TFD) % 8 == 0,
              "TMA destinations must be 128-byte aligned");
// the tensor maps of one launch: spinor boxes (centre, x, y, t faces) and link boxes
struct alignas(64) Maps {
  CUtensorMap cen, xf, yf, tf, ut, ux, uy, utm;
};
constexpr unsigned long long kWaitNs = 200000000ull;  // bound on each mbarrier wait: 0.2 s of global time
}  // namespace tile

// blocks of the staged-tile stencil whose copies did not arrive within the bound (per device);
// read by thr_stencil_timeouts
__device__ unsigned long long g_stencil_timeouts = 0;

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// polls the mbarrier until the phase of the given parity completes or kWaitNs have passed;
// 1 if it completed
__device__ __forceinline__ unsigned mbar_wait_bounded(unsigned bar, unsigned parity = 0) {
  unsigned done = 0;
  const unsigned long long t0 = global_ns();
  for (unsigned k = 0; !done; k++) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (!done && (k & 63) == 63 && global_ns() - t0 > tile::kWaitNs) break;
  }
  return done;
}

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void tma_load5(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4,
                                          unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], "
      "[%7];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4),
      "r"(smem_u32(bar))
      : "memory");
}

// thread 0 of a block: the 11 tensor copies of the tile at (x0, y0, t0, s0) into sm, all
// completing on `bar` (expecting `bytes`)
__device__ __forceinline__ void tile_issue(double2* sm, const tile::Maps& maps, unsigned long long* bar,
                                           const Geom& g, int x0, int y0, int t0, int s0, int bytes) {
  using namespace tile;
  const int Lx = g.lx, Ly = g.ly, Lt = g.lt;
  const int xm = x0 == 0 ? Lx - 1 : x0 - 1, xp = x0 + TX == Lx ? 0 : x0 + TX;
  const int ym = y0 == 0 ? Ly - 1 : y0 - 1, yp = y0 + TY == Ly ? 0 : y0 + TY;
  const int tm = t0 == 0 ? Lt - 1 : t0 - 1, tp = t0 + TT == Lt ? 0 : t0 + TT;
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
  const int c0 = 2 * s0;  // fifth-dimension coordinate in doubles: 16-byte multiples
  tma_load5(sm + CEN, &maps.cen, c0 - 2, x0, y0, t0, 0, bar);
  tma_load5(sm + XF, &maps.xf, c0, xm, y0, t0, 0, bar);
  tma_load5(sm + XF + 4 * XFD, &maps.xf, c0, xp, y0, t0, 0, bar);
  tma_load5(sm + YF, &maps.yf, c0, x0, ym, t0, 0, bar);
  tma_load5(sm + YF + 4 * YFD, &maps.yf, c0, x0, yp, t0, 0, bar);
  tma_load5(sm + TF, &maps.tf, c0, x0, y0, tm, 0, bar);
  tma_load5(sm + TF + 4 * TFD, &maps.tf, c0, x0, y0, tp, 0, bar);
  tma_load5(sm + UT, &maps.ut, 0, x0, y0, t0, 0, bar);
  tma_load5(sm + UX, &maps.ux, 0, xm, y0, t0, 0, bar);
  tma_load5(sm + UY, &maps.uy, 0, x0, ym, t0, 1, bar);
  tma_load5(sm + UTM, &maps.utm, 0, x0, y0, tm, 2, bar);
}

// shamir_site's arithmetic, operation for operation, for the thread's 5D site (s = s0 + sl
// at tile position xs, ys, ts) with every operand from the staged tile sm
template <bool DAG>
__device__ __forceinline__ void tile_site(const double2* sm, int Ls, int s, int sl, int xs, int ys, int ts,
                                          float am, int imass, float am3, double2* acc) {
  using namespace tile;
  const int q = (ts * TY + ys) * TX + xs;  // tile site
  constexpr int CD = NS * CW;              // centre: stride of the spin index
  const double2* cen = sm + CEN + q * CW + sl + 1;  // R(s) of spin 0 at this site
  const double diag = (double)((3.0f - am3) + 1.0f);  // dirac.F90:45, default real
  double2 rc[4];
#pragma unroll
  for (int d = 0; d < 4; d++) {
    rc[d] = cen[d * CD];
    acc[d] = diag * rc[d];
  }
  // fifth dimension and walls as in shamir_site: the slot after s holds R(s+1),
  // or R(0) at s = Ls-1; the slot before s holds R(s-1), or R(Ls-1) at s = 0
  const int a0 = DAG ? 0 : 2, b0 = DAG ? 2 : 0;
#pragma unroll
  for (int k = 0; k < 2; k++) {
    if (s < Ls - 1) acc[a0 + k] = acc[a0 + k] - cen[(a0 + k) * CD + 1];
    if (s > 0) acc[b0 + k] = acc[b0 + k] - cen[(b0 + k) * CD - 1];
  }
  const double a = (double)am;
  const bool five = imass == 5;
  const double2 cA = imass == 1 ? mk(a, 0.0) : mk(0.0, (five && DAG) ? -a : a);
  const double2 cB = imass == 1 ? mk(a, 0.0) : mk(0.0, five ? (DAG ? -a : a) : -a);
#pragma unroll
  for (int k = 0; k < 2; k++) {
    if (s == Ls - 1) acc[a0 + k] = acc[a0 + k] + cmul(cA, five ? rc[b0 + k] : cen[(a0 + k) * CD + 1]);
    if (s == 0) acc[b0 + k] = acc[b0 + k] + cmul(cB, five ? rc[a0 + k] : cen[(b0 + k) * CD - 1]);
  }
  // hops in shamir_site's order: per direction forward then backward
#pragma unroll
  for (int mu = 0; mu < 3; mu++) {
#pragma unroll
    for (int dir = 0; dir < 2; dir++) {
      const double2* p;
      int dstr;
      double2 W;
      if (mu == 0) {
        const bool in_tile = dir == 0 ? xs < TX - 1 : xs > 0;
        p = in_tile ? cen + (dir == 0 ? CW : -CW) : sm + XF + (dir == 0 ? 4 * XFD : 0) + (ts * TY + ys) * SC + sl;
        dstr = in_tile ? CD : XFD;
        W = dir == 0 ? sm[UT + q] : cconj(xs > 0 ? sm[UT + q - 1] : sm[UX + ts * TY + ys]);
      } else if (mu == 1) {
        const bool in_tile = dir == 0 ? ys < TY - 1 : ys > 0;
        p = in_tile ? cen + (dir == 0 ? TX * CW : -TX * CW)
                    : sm + YF + (dir == 0 ? 4 * YFD : 0) + (ts * TX + xs) * SC + sl;
        dstr = in_tile ? CD : YFD;
        W = dir == 0 ? sm[UT + NS + q] : cconj(ys > 0 ? sm[UT + NS + q - TX] : sm[UY + ts * TX + xs]);
      } else {
        const bool in_tile = dir == 0 ? ts < TT - 1 : ts > 0;
        p = in_tile ? cen + (dir == 0 ? TY * TX * CW : -TY * TX * CW)
                    : sm + TF + (dir == 0 ? 4 * TFD : 0) + (ys * TX + xs) * SC + sl;
        dstr = in_tile ? CD : TFD;
        W = dir == 0 ? sm[UT + 2 * NS + q] : cconj(ts > 0 ? sm[UT + 2 * NS + q - TY * TX] : sm[UTM + ys * TX + xs]);
      }
      double2 r[4];
#pragma unroll
      for (int d = 0; d < 4; d++) r[d] = p[d * dstr];
      hop_projected<double2, double>(mu, (dir == 0) != DAG, W, r, acc);
    }
  }
}

template <bool DAG, int EPI>
__global__ void __launch_bounds__(tile::NT, 4)
    k_dslash_tile(double2* __restrict__ out, const double2* __restrict__ in, const __grid_constant__ tile::Maps maps,
                  Geom g, float am, int imass, float am3, const int* skip, const double2* __restrict__ aux,
                  const double* __restrict__ coef, double* __restrict__ partials, int rev, int extra_tx) {
  using namespace tile;
  if (skip && *skip) return;
  // the dynamic region is allocated 128 bytes long and rounded up to a 128-byte
  // boundary of the shared window, where TMA destinations must start
  extern __shared__ __align__(16) double2 smraw[];
  double2* const sm = smraw + ((128u - (smem_u32(smraw) & 127u)) & 127u) / 16u;
  __shared__ __align__(8) unsigned long long bar;
  const int Lx = g.lx, Ly = g.ly, Lt = g.lt, Ls = g.ls;
  const unsigned v3 = (unsigned)g.v3;
  const int nch = Ls / SC;
  // rev: blocks walk the tiles from the top (see k_dslash)
  const int bid = rev ? (int)gridDim.x - 1 - (int)blockIdx.x : (int)blockIdx.x;
  const int ch = bid % nch, ti = bid / nch;
  const int ntx = Lx / TX, nty = Ly / TY;
  const int x0 = (ti % ntx) * TX, y0 = ((ti / ntx) % nty) * TY, t0 = (ti / (ntx * nty)) * TT, s0 = ch * SC;
  const int tid = threadIdx.x;
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) tile_issue(sm, maps, &bar, g, x0, y0, t0, s0, END * (int)sizeof(double2) + extra_tx);
  // wall values for the s-neighbour slots outside the tensor: R(Ls-1) before s = 0
  // (threads 0-127, one centre row each) and R(0) after s = Ls-1 (threads 128-255)
  const int row = tid & 127;
  const bool wall = tid < 128 ? ch == 0 : ch == nch - 1;
  double2 wv = mk(0.0, 0.0);
  if (wall) {
    const unsigned wsite = (unsigned)(x0 + (row & 3) + Lx * (y0 + ((row >> 2) & 3) + Ly * (t0 + ((row >> 4) & 1))));
    wv = in[(unsigned)(tid < 128 ? Ls - 1 : 0) + (unsigned)Ls * (wsite + v3 * (unsigned)(row >> 5))];
  }
  const unsigned done = mbar_wait_bounded(smem_u32(&bar));
  if (wall) sm[CEN + row * CW + (tid < 128 ? 0 : CW - 1)] = wv;
  const int sl = tid & 7, xs = (tid >> 3) & 3, ys = (tid >> 5) & 3, ts = tid >> 7;
  const int s = s0 + sl;
  const unsigned site = (unsigned)(x0 + xs + Lx * (y0 + ys + Ly * (t0 + ts)));
  if (!__syncthreads_and(done)) {
    // The copies did not all arrive within the bound.  One more bounded wait, so that no
    // copy still writes this block's shared memory when the block exits (if that wait
    // also runs out, the block exits anyway); the event is counted for the host
    // (thr_stencil_timeouts) and every output of the block, and its partial, become NaN,
    // whichever epilogue runs, so that every caller sees the failure.
    if (tid == 0) {
      mbar_wait_bounded(smem_u32(&bar));
      atomicAdd(&g_stencil_timeouts, 1ull);
    }
    const double qnan = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
    for (int d = 0; d < 4; d++) out[(unsigned)s + (unsigned)Ls * (site + v3 * (unsigned)d)] = mk(qnan, qnan);
    if (EPI != 0 && tid == 0) partials[bid] = qnan;
    __syncthreads();
    return;
  }

  const double om = (EPI == 1 || EPI == 3) ? *coef : 0.0;
  double2 acc[4];
  tile_site<DAG>(sm, Ls, s, sl, xs, ys, ts, am, imass, am3, acc);
  double racc = 0.0;
#pragma unroll
  for (int d = 0; d < 4; d++) {
    const unsigned i = (unsigned)s + (unsigned)Ls * (site + v3 * (unsigned)d);
    if (EPI == 1) {
      const double2 rn = aux[i] + om * acc[d];  // r = r + omega*s (multishift_module.F90:137)
      out[i] = rn;
      racc += epi_norm<double2>(rn);
    } else if (EPI == 3) {
      const double2 hn = acc[d] + om * aux[i];  // h = M r + gamma h (= M p by linearity)
      out[i] = hn;
      racc += epi_norm<double2>(hn);
    } else {
      out[i] = acc[d];
      if (EPI == 2) racc += epi_norm<double2>(acc[d]);
    }
  }
  if (EPI != 0) {
    // one FP64 partial per block, fixed order: warp sums, then the 8 warps in turn
    __shared__ double red[NT / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) racc += __shfl_down_sync(0xffffffffu, racc, o);
    if ((tid & 31) == 0) red[tid >> 5] = racc;
    __syncthreads();
    if (tid == 0) {
      double v = 0.0;
#pragma unroll
      for (int w = 0; w < NT / 32; w++) v += red[w];
      partials[bid] = v;
    }
  }
}

// Persistent double-buffered form of the staged-tile stencil.  A block walks the tiles
// blockIdx.x, blockIdx.x + gridDim.x, ... with two tile buffers: while it computes tile k
// from one, the copies of tile k + 1 land in the other, and the wall values and the
// epilogue's operand are loaded before the wait, so copies, arithmetic and stores of a block
// overlap (2 blocks of 2 x 54 KB per SM).  Tile numbering, arithmetic (tile_site), the
// per-tile partial sums and their order are k_dslash_tile's, so the results are its bits.
constexpr int kTile2PerSm = 2;
constexpr int kTile2Buf = ((tile::END + 7) / 8) * 8;  // buffer stride in double2 (a 128-byte multiple)
constexpr int kTile2Smem = 2 * kTile2Buf * (int)sizeof(double2) + 128;

template <bool DAG, int EPI>
__global__ void __launch_bounds__(tile::NT, kTile2PerSm)
    k_dslash_tile2(double2* __restrict__ out, const double2* __restrict__ in, const __grid_constant__ tile::Maps maps,
                   Geom g, float am, int imass, float am3, const int* skip, const double2* __restrict__ aux,
                   const double* __restrict__ coef, double* __restrict__ partials, int rev, int extra_tx) {
  using namespace tile;
  if (skip && *skip) return;
  extern __shared__ __align__(16) double2 smraw[];
  double2* const smb = smraw + ((128u - (smem_u32(smraw) & 127u)) & 127u) / 16u;
  __shared__ __align__(8) unsigned long long bar[2];
  __shared__ double red[NT / 32];
  const int Lx = g.lx, Ly = g.ly, Ls = g.ls;
  const unsigned v3 = (unsigned)g.v3;
  const int nch = Ls / SC;
  const int ntiles = (int)(v3 / (unsigned)NS) * nch;
  const int ntx = Lx / TX, nty = Ly / TY;
  const int tid = threadIdx.x;
  const int bytes = END * (int)sizeof(double2) + extra_tx;
  // tile -> its index in k_dslash_tile's numbering (rev: from the top) and its origin
  auto origin = [&](int tl, int& bid, int& ch, int& x0, int& y0, int& t0, int& s0) {
    bid = rev ? ntiles - 1 - tl : tl;
    ch = bid % nch;
    const int ti = bid / nch;
    x0 = (ti % ntx) * TX;
    y0 = ((ti / ntx) % nty) * TY;
    t0 = (ti / (ntx * nty)) * TT;
    s0 = ch * SC;
  };
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&bar[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&bar[1])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  int tl = blockIdx.x;
  if (tid == 0 && tl < ntiles) {
    int b0_, c_, x_, y_, t_, s_;
    origin(tl, b0_, c_, x_, y_, t_, s_);
    tile_issue(smb, maps, &bar[0], g, x_, y_, t_, s_, bytes);
  }
  const double om = (EPI == 1 || EPI == 3) ? *coef : 0.0;
  const int sl = tid & 7, xs = (tid >> 3) & 3, ys = (tid >> 5) & 3, ts = tid >> 7;
  const int row = tid & 127;
  for (int k = 0; tl < ntiles; k++, tl += gridDim.x) {
    const int b = k & 1;
    double2* const sm = smb + b * kTile2Buf;
    int bid, ch, x0, y0, t0, s0;
    origin(tl, bid, ch, x0, y0, t0, s0);
    const int next = tl + (int)gridDim.x;
    if (tid == 0 && next < ntiles) {
      // the other buffer was last read in iteration k - 1, which ended in a barrier: order
      // those accesses before the copies that overwrite it
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      int nb, nc, nx0, ny0, nt0, ns0;
      origin(next, nb, nc, nx0, ny0, nt0, ns0);
      tile_issue(smb + (b ^ 1) * kTile2Buf, maps, &bar[b ^ 1], g, nx0, ny0, nt0, ns0, bytes);
    }
    const int s = s0 + sl;
    const unsigned site = (unsigned)(x0 + xs + Lx * (y0 + ys + Ly * (t0 + ts)));
    // the wall values (R(Ls-1) before s = 0, R(0) after s = Ls-1) and the epilogue's operand,
    // loaded while this tile's copies may still be in flight
    const bool wall = tid < 128 ? ch == 0 : ch == nch - 1;
    double2 wv = mk(0.0, 0.0);
    if (wall) {
      const unsigned wsite =
          (unsigned)(x0 + (row & 3) + Lx * (y0 + ((row >> 2) & 3) + Ly * (t0 + ((row >> 4) & 1))));
      wv = in[(unsigned)(tid < 128 ? Ls - 1 : 0) + (unsigned)Ls * (wsite + v3 * (unsigned)(row >> 5))];
    }
    double2 av[4];
#pragma unroll
    for (int d = 0; d < 4; d++)
      av[d] = (EPI == 1 || EPI == 3) ? aux[(unsigned)s + (unsigned)Ls * (site + v3 * (unsigned)d)] : mk(0.0, 0.0);
    const unsigned done = mbar_wait_bounded(smem_u32(&bar[b]), (unsigned)(k >> 1) & 1u);
    if (wall) sm[CEN + row * CW + (tid < 128 ? 0 : CW - 1)] = wv;
    if (!__syncthreads_and(done)) {
      // The copies did not all arrive within the bound.  Bounded waits for this tile's and
      // the next tile's copies, so that none still lands in shared memory when the block
      // exits (if they run out too, the block exits anyway); the event is counted for the
      // host (thr_stencil_timeouts), and this and every later tile of the block get NaN
      // outputs and partials, whichever epilogue runs.
      if (tid == 0) {
        if (next < ntiles) mbar_wait_bounded(smem_u32(&bar[b ^ 1]), (unsigned)((k + 1) >> 1) & 1u);
        mbar_wait_bounded(smem_u32(&bar[b]), (unsigned)(k >> 1) & 1u);
        atomicAdd(&g_stencil_timeouts, 1ull);
      }
      const double qnan = __longlong_as_double(0x7ff8000000000000LL);
      for (int t2 = tl; t2 < ntiles; t2 += gridDim.x) {
        int b2, c2, x2, y2, tt2, s2;
        origin(t2, b2, c2, x2, y2, tt2, s2);
        const unsigned st2 = (unsigned)(x2 + xs + Lx * (y2 + ys + Ly * (tt2 + ts)));
#pragma unroll
        for (int d = 0; d < 4; d++) out[(unsigned)(s2 + sl) + (unsigned)Ls * (st2 + v3 * (unsigned)d)] = mk(qnan, qnan);
        if (EPI != 0 && tid == 0) partials[b2] = qnan;
      }
      __syncthreads();
      return;
    }
    double2 acc[4];
    tile_site<DAG>(sm, Ls, s, sl, xs, ys, ts, am, imass, am3, acc);
    double racc = 0.0;
#pragma unroll
    for (int d = 0; d < 4; d++) {
      const unsigned i = (unsigned)s + (unsigned)Ls * (site + v3 * (unsigned)d);
      if (EPI == 1) {
        const double2 rn = av[d] + om * acc[d];  // r = r + omega*s (multishift_module.F90:137)
        out[i] = rn;
        racc += epi_norm<double2>(rn);
      } else if (EPI == 3) {
        const double2 hn = acc[d] + om * av[d];  // h = M r + gamma h (= M p by linearity)
        out[i] = hn;
        racc += epi_norm<double2>(hn);
      } else {
        out[i] = acc[d];
        if (EPI == 2) racc += epi_norm<double2>(acc[d]);
      }
    }
    if (EPI != 0) {
      // one FP64 partial per tile, the order of k_dslash_tile: warp sums, then the 8 warps in turn
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) racc += __shfl_down_sync(0xffffffffu, racc, o);
      if ((tid & 31) == 0) red[tid >> 5] = racc;
      __syncthreads();
      if (tid == 0) {
        double v = 0.0;
#pragma unroll
        for (int w = 0; w < NT / 32; w++) v += red[w];
        partials[bid] = v;
      }
    }
    __syncthreads();  // this buffer and red[] are free for the next iteration
  }
}

// Tensor maps of the staged-tile kernel for the spinor field `in` and the links u
// (cuTensorMapEncodeTiled through the runtime's driver entry point; the maps are
// plain host structures passed by value, so graphs capture them with the launch)
namespace {
using EncodeFn = PFN_cuTensorMapEncodeTiled_v12000;
EncodeFn tile_encoder() {
  static EncodeFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<EncodeFn>(p);
  }();
  return fn;
}
bool tile_map(EncodeFn enc, CUtensorMap* m, const void* base, const cuuint64_t* dim, const cuuint64_t* stride,
              const cuuint32_t* box) {
  const cuuint32_t es[5] = {1, 1, 1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, const_cast<void*>(base), dim, stride, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
bool tile_maps(const Geom& g, const double2* in, const double2* u, tile::Maps* m) {
  using namespace tile;
  const EncodeFn enc = tile_encoder();
  if (!enc) return false;
  const cuuint64_t row = 16ull * g.ls;  // bytes of one (site, spin) run of the fifth dimension
  const cuuint64_t sd[5] = {2ull * g.ls, (cuuint64_t)g.lx, (cuuint64_t)g.ly, (cuuint64_t)g.lt, 4};
  const cuuint64_t ss[4] = {row, row * g.lx, row * g.lx * g.ly, row * g.v3};
  const cuuint64_t ud[5] = {2, (cuuint64_t)g.lx, (cuuint64_t)g.ly, (cuuint64_t)g.lt, 3};
  const cuuint64_t us[4] = {16, 16ull * g.lx, 16ull * g.lx * g.ly, 16ull * g.v3};
  const cuuint32_t bc[5] = {2 * CW, TX, TY, TT, 4}, bx[5] = {2 * SC, 1, TY, TT, 4}, by[5] = {2 * SC, TX, 1, TT, 4},
                   bt[5] = {2 * SC, TX, TY, 1, 4};
  const cuuint32_t ut[5] = {2, TX, TY, TT, 3}, ux[5] = {2, 1, TY, TT, 1}, uy[5] = {2, TX, 1, TT, 1},
                   utm[5] = {2, TX, TY, 1, 1};
  return tile_map(enc, &m->cen, in, sd, ss, bc) && tile_map(enc, &m->xf, in, sd, ss, bx) &&
         tile_map(enc, &m->yf, in, sd, ss, by) && tile_map(enc, &m->tf, in, sd, ss, bt) &&
         tile_map(enc, &m->ut, u, ud, us, ut) && tile_map(enc, &m->ux, u, ud, us, ux) &&
         tile_map(enc, &m->uy, u, ud, us, uy) && tile_map(enc, &m->utm, u, ud, us, utm);
}
}  // namespace

// Batched stencil: a persistent grid walks the work blocks of all entries
// (right-hand sides or lattices).  Work block wb belongs to the entry e with
// blk0[e] <= wb < blk0[e+1]; inside it, thread tid handles s = tid % Ls of
// site (wb - blk0) * spb + tid / Ls.  Entries with skip[e] set are passed over.
// EPI: 0 out = M in; 1 also a partial of Re<aux, M in> per work block; 2 also a partial
// of |M in|^2; 4 the CG residual update fused in: rv -= coef_e (M in) in place, in the
// arithmetic type, with a partial of |rv|^2 (coef_e = coef[e * coef_stride], the entry's
// own CG scalar; out is not written)
template <class S, int KER, bool DAG, int EPI>
__global__ void __launch_bounds__(256, KER == 0 ? 4 : 1)
    k_dslash_batch(S* __restrict__ out, const S* __restrict__ in, const typename Sto<S>::C* __restrict__ u,
                   const BatchEntry* __restrict__ tab, int nent, int total_blocks, float am, int imass, float am3,
                   const int* skip, const S* __restrict__ aux, double* __restrict__ partials,
                   typename Sto<S>::C* rv, const double* coef, int coef_stride) {
  using C = typename Sto<S>::C;
  using R = typename Sto<S>::R;
  for (int wb = blockIdx.x; wb < total_blocks; wb += gridDim.x) {
    int lo = 0, hi = nent - 1;  // last entry with blk0 <= wb
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (tab[mid].blk0 <= wb) lo = mid;
      else hi = mid - 1;
    }
    const BatchEntry& E = tab[lo];
    if (skip && skip[lo]) continue;
    const Geom g = E.g;
    const int s = threadIdx.x % g.ls;
    const int sub = threadIdx.x / g.ls;
    const int site = (wb - E.blk0) * E.spb + sub;
    double racc = 0.0;
    if (sub < E.spb && site < g.v3) {
      C acc[4];
      apply_site<S, KER, DAG>(in + E.off, u + E.uoff, g, s, site, am, imass, am3, acc);
      if (EPI == 4) {
        const R a = (R)coef[(size_t)lo * coef_stride];
        C* r = rv + E.off;
#pragma unroll
        for (int d = 0; d < 4; d++) {
          const size_t i = sidx(g, s, site, d);
          const C rn = r[i] - a * acc[d];  // r = r - alpha M^dagger M p (measure_module.F90:92)
          r[i] = rn;
          racc += epi_norm<S>(rn);
        }
      } else {
#pragma unroll
        for (int d = 0; d < 4; d++) {
          Sto<S>::st(out + E.off, sidx(g, s, site, d), acc[d]);
          if (EPI == 1) racc += epi_redot<S>(aux + E.off, sidx(g, s, site, d), acc[d]);
          if (EPI == 2) racc += epi_norm<S>(acc[d]);
        }
      }
    }
    if (EPI != 0) block_partial(racc, partials + wb);
  }
}

// ---------------------------------------------------------------- launch
int device_sms() {
  constexpr int kDevs = 64;
  static std::atomic<int> cache[kDevs];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 148;
  if (dev < kDevs) {
    const int v = cache[dev].load(std::memory_order_relaxed);
    if (v > 0) return v;
  }
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 148;
  if (dev < kDevs) cache[dev].store(sms, std::memory_order_relaxed);
  return sms;
}

namespace {
int stencil_threads(const Geom& g, int kernel) {
  const int nt = kernel == 0 ? 128 : 256;
  return g.ls <= nt ? nt : 1024;
}
bool stencil_shfl(const Geom& g, int kernel) { return kernel == 0 && g.ls <= 32 && (g.ls & (g.ls - 1)) == 0; }
// THR_TILE=1 in the environment puts the FP64 Shamir stencil on the staged-tile
// kernel where the lattice allows it.  It is off by default: on B200 it measured
// 51-54 us per launch in the 32^2x32, Ls 32 multishift solve against k_dslash's
// 48-50 us, and 162 us against 156-159 us at 48^2x48, Ls 48.
// THR_TILE: 1 the staged-tile kernel, 2 its persistent double-buffered form
int tile_mode() {
  static const int mode = [] {
    const char* e = std::getenv("THR_TILE");
    return (e && (e[0] == '1' || e[0] == '2') && e[1] == 0) ? e[0] - '0' : 0;
  }();
  return mode;
}
bool tile_on() { return tile_mode() != 0; }
// THR_TILE_WAIT_TEST=1 (with THR_TILE=1) makes the staged-tile kernel expect 16 bytes more
// than its copies bring, so that its bounded wait runs out with every copy already complete:
// a test of the timeout path (NaN outputs, thr_stencil_timeouts) that faults nothing
int tile_extra_tx() {
  static const int extra = [] {
    const char* e = std::getenv("THR_TILE_WAIT_TEST");
    return e && e[0] == '1' && e[1] == 0 ? 16 : 0;
  }();
  return extra;
}
bool tile_ok(const Geom& g, int kernel) {
  return kernel == 0 && g.layout != LAYOUT_EO && g.lx % tile::TX == 0 && g.ly % tile::TY == 0 &&
         g.lt % tile::TT == 0 && g.ls % tile::SC == 0 && tile_on();
}
unsigned tile_grid(const Geom& g) { return (unsigned)(g.v3 / tile::NS) * (unsigned)(g.ls / tile::SC); }
}  // namespace

unsigned stencil_parts(const Geom& g, int kernel, bool fp64) {
  return fp64 && tile_ok(g, kernel) ? tile_grid(g) : stencil_grid(g, kernel);
}

dim3 stencil_block(const Geom& g, int kernel) {
  int spb = stencil_threads(g, kernel) / g.ls;
  if (spb < 1) spb = 1;
  return dim3(g.ls, spb, 1);
}

// one block row per site: ceil(V3 / sites per block) blocks (each writes one
// partial when an epilogue reduction is requested)
unsigned stencil_grid(const Geom& g, int kernel) {
  const dim3 blk = stencil_block(g, kernel);
  return (unsigned)((g.v3 + blk.y - 1) / blk.y);
}

// ---------------------------------------------------------------- autotuner
// For the stencils in FP64 and FP32 storage the register budget (blocks per SM
// the compiler may assume: 8, 7 or 6 for the Shamir kernel's 128-thread blocks,
// 4, 3 or 2 for the Wilson kernel's 256-thread blocks) is tuned per (storage,
// kernel, M or M^dagger, epilogue, lattice, layout, device) on first use:
// each candidate runs 1 + 3 times on the call's own fields (the launches are
// idempotent: out and partials are overwritten), the fastest is kept for the
// process.  For the FP64 Shamir stencil the candidates also vary the threads
// per site (k_dslash_split, 40), the sites per block (k_dslash_g2: 2, 4 or 8
// k_dslash blocks in one, 224, 223, 242, 281) and, with Ls a power of two <= 32,
// whether the fifth dimension comes
// from warp shuffles or from memory (108, 106); every candidate computes each
// output element with the same operations
// and sums the partials over the same site groups in the same order, so the
// results do not change.  THR_TUNE=0 in the environment keeps the defaults
// (8, 4); THR_TUNE=<n> runs candidate n wherever it is one.  Launches made
// while the stream is being captured into a graph use the default until a
// tuned value exists.
namespace {
constexpr int kTuneShamir[3] = {8, 7, 6};
// FP64 storage adds the four-threads-per-site kernel (k_dslash_split) as a candidate
constexpr int kSplitCode = 40;
// and, where a block's Ls x sites threads are whole warps, blocks of K site groups
// (k_dslash_g2): K = 2 at 4 or 3 resident blocks per SM, K = 4 at 2, K = 8 at 1:
// candidates kG2Code + 10 K + MINB
constexpr int kG2Code = 200;
// and, where the fifth dimension comes from warp shuffles (Ls a power of two <= 32), the
// same kernel reading the fifth-dimension neighbours from memory instead (the same
// values, so the same bits): candidates kNoShflCode + 8, kNoShflCode + 6
constexpr int kNoShflCode = 100;
constexpr int kTuneWilson[3] = {4, 3, 2};
constexpr int kTuneOverlap[3] = {4, 3, 1};  // k_odslash's 256-thread blocks
constexpr int kMaxCand = 10;
struct TuneKey {
  int dev, sid, ker, dag, epi, lx, ly, lt, ls, layout;
  bool operator<(const TuneKey& o) const {
    const int a[10] = {dev, sid, ker, dag, epi, lx, ly, lt, ls, layout};
    const int b[10] = {o.dev, o.sid, o.ker, o.dag, o.epi, o.lx, o.ly, o.lt, o.ls, o.layout};
    for (int i = 0; i < 10; i++)
      if (a[i] != b[i]) return a[i] < b[i];
    return false;
  }
};
struct TuneVal {
  int pick, ncand;
  float us[kMaxCand];
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneVal> g_tune;
int g_tune_mode = -1;  // -1: not read yet, 0 off, 1 on
int g_tune_force = 0;  // THR_TUNE=<candidate code>: that candidate wherever it is one
bool tune_on() {
  if (g_tune_mode < 0) {
    const char* e = std::getenv("THR_TUNE");
    g_tune_mode = (e && e[0] == '0') ? 0 : 1;
    if (e && std::atoi(e) >= 2) g_tune_force = std::atoi(e);
  }
  return g_tune_mode == 1;
}
bool capturing(cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) return true;
  return cs != cudaStreamCaptureStatusNone;
}
template <class S> constexpr int storage_id() { return sizeof(S) == sizeof(double2) ? 0 : sizeof(S) == sizeof(float2) ? 1 : 2; }
}  // namespace

// the tuned candidate for `key`: looked up, forced by THR_TUNE=<n>, or timed now
// (each candidate 1 + 3 launches on the call's own fields) unless the stream is
// being captured; cand[0] when tuning is off or cannot run
template <class F>
int tune_pick(const TuneKey& key, const int* cand, int ncand, cudaStream_t st, F&& launch) {
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) return it->second.pick;
  }
  if (!tune_on()) return cand[0];
  if (g_tune_force) {
    for (int c = 0; c < ncand; c++)
      if (cand[c] == g_tune_force) return g_tune_force;
    return cand[0];
  }
  if (capturing(st)) return cand[0];
  TuneVal tv{cand[0], ncand, {}};
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return cand[0];
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return cand[0];
  }
  float best = 1e30f;
  for (int c = 0; c < ncand; c++) {
    launch(cand[c]);
    cudaEventRecord(e0, st);
    for (int r = 0; r < 3; r++) launch(cand[c]);
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    tv.us[c] = ms * 1e3f / 3.f;
    if (tv.us[c] < best) {
      best = tv.us[c];
      tv.pick = cand[c];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tune[key] = tv;
  return tv.pick;
}

// the candidate already tuned for `key`, else cand[0]; never times anything
int tune_lookup(const TuneKey& key, const int* cand) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  auto it = g_tune.find(key);
  return it != g_tune.end() ? it->second.pick : cand[0];
}

// epi: 0 none, 1 out = aux + (*coef) M in with |out|^2 per block, 2 |out|^2 per block
// may_tune false: no timing launches and no events (a budget tuned earlier is still used)
template <class S>
int launch_dslash_mode(const Geom& g, int kernel, bool dag, S* out, const S* in, const typename Sto<S>::C* u, float am,
                       int imass, float am3, cudaStream_t st, const int* skip, const S* aux, const double* coef,
                       double* partials, int e, int rev, bool may_tune = true, bool pdl = false) {
  if (g.ls > 1024) return THR_ERR_BADSHAPE;
  if (4ULL * (unsigned long long)g.v5 >= (1ULL << 32)) return THR_ERR_BADSHAPE;  // 32-bit element offsets
  if (kernel == 1 && imass != 1 && imass != 3) return THR_ERR_UNSUPPORTED;  // dwf3d_lib.F90:152-158
  if (storage_id<S>() == 0 && tile_ok(g, kernel)) {
    double2* o = reinterpret_cast<double2*>(out);
    const double2* i = reinterpret_cast<const double2*>(in);
    const double2* ax = reinterpret_cast<const double2*>(aux);
    const unsigned grd = tile_grid(g);
    const unsigned grd2 = std::min(grd, (unsigned)(kTile2PerSm * device_sms()));
    tile::Maps maps;
    if (!tile_maps(g, i, reinterpret_cast<const double2*>(u), &maps)) return THR_ERR_CUDA;
    int dev = 0;
    cudaGetDevice(&dev);
#define THR_T(D, E)                                                                                          \
  do {                                                                                                       \
    static std::atomic<unsigned long long> attr{0}; /* devices whose attributes are set */                 \
    if (dev >= 64 || !(attr.load() >> dev & 1ull)) {                                                         \
      cudaFuncSetAttribute(k_dslash_tile<D, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, tile::SMEM);    \
      cudaFuncSetAttribute(k_dslash_tile<D, E>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);        \
      cudaFuncSetAttribute(k_dslash_tile2<D, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTile2Smem);   \
      cudaFuncSetAttribute(k_dslash_tile2<D, E>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);       \
      if (dev < 64) attr.fetch_or(1ull << dev);                                                              \
    }                                                                                                        \
    if (tile_mode() == 2)                                                                                    \
      k_dslash_tile2<D, E><<<grd2, tile::NT, kTile2Smem, st>>>(o, i, maps, g, am, imass, am3, skip, ax, coef, \
                                                               partials, rev, tile_extra_tx());              \
    else                                                                                                     \
      k_dslash_tile<D, E><<<grd, tile::NT, tile::SMEM, st>>>(o, i, maps, g, am, imass, am3, skip, ax, coef,   \
                                                             partials, rev, tile_extra_tx());                \
  } while (0)
#define THR_TE(D)                 \
  do {                            \
    if (e == 1) THR_T(D, 1);      \
    else if (e == 2) THR_T(D, 2); \
    else if (e == 3) THR_T(D, 3); \
    else THR_T(D, 0);             \
  } while (0)
    if (dag) THR_TE(true);
    else THR_TE(false);
#undef THR_TE
#undef THR_T
    return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
  }
  const dim3 blk = stencil_block(g, kernel);
  const dim3 grd(stencil_grid(g, kernel));
  const int nt = stencil_threads(g, kernel);
  const bool shfl = stencil_shfl(g, kernel);
#define THR_L(K, D, E, N, SH, MB)                                                                           \
  launch_k(k_dslash<S, K, D, E, N, SH, MB>, grd, blk, 0, st, pdl, out, in, u, g, am, imass, am3, skip, aux, coef, \
           partials, rev)
#define THR_E(K, D, N, SH, MB)                 \
  do {                                         \
    if (e == 1) THR_L(K, D, 1, N, SH, MB);     \
    else if (e == 2) THR_L(K, D, 2, N, SH, MB); \
    else if (e == 3) THR_L(K, D, 3, N, SH, MB); \
    else THR_L(K, D, 0, N, SH, MB);            \
  } while (0)
#define THR_D(K, N, SH, MB)                        \
  do {                                             \
    if (dag) THR_E(K, true, N, SH, MB);            \
    else THR_E(K, false, N, SH, MB);               \
  } while (0)
  // FP32 Shamir with even Ls: two s per thread (k_dslash_pair), same grid
  const bool pair = storage_id<S>() == 1 && kernel == 0 && nt == 128 && g.ls % 2 == 0;

  // the register budget (resident blocks per SM) of the common configurations is
  // tuned: Shamir 128-thread blocks {8, 7, 6} (pair kernel: 64-thread blocks {16, 14, 12}),
  // Wilson 256-thread blocks {2, 1}
  auto launch = [&](int minb) {
    if (pair) {
      const dim3 pblk(g.ls / 2, blk.y, 1);
      const float2* in2 = reinterpret_cast<const float2*>(in);
      float2* out2 = reinterpret_cast<float2*>(out);
      const float2* aux2 = reinterpret_cast<const float2*>(aux);
      const float2* u2 = reinterpret_cast<const float2*>(u);
#define THR_P(D, E, MB)                                                                                     \
  launch_k(k_dslash_pair<float2, D, E, MB>, grd, pblk, 0, st, pdl, out2, in2, u2, g, am, imass, am3, skip, aux2, \
           coef, partials, rev)
#define THR_PE(D, MB)                    \
  do {                                   \
    if (e == 1) THR_P(D, 1, MB);         \
    else if (e == 2) THR_P(D, 2, MB);    \
    else if (e == 3) THR_P(D, 3, MB);    \
    else THR_P(D, 0, MB);                \
  } while (0)
      const int mb = minb == 8 ? 16 : minb == 7 ? 14 : 12;
      if (dag) {
        if (mb == 16) THR_PE(true, 16);
        else if (mb == 14) THR_PE(true, 14);
        else THR_PE(true, 12);
      } else {
        if (mb == 16) THR_PE(false, 16);
        else if (mb == 14) THR_PE(false, 14);
        else THR_PE(false, 12);
      }
#undef THR_PE
#undef THR_P
      return;
    }
    if (kernel == 1) {
      // Ls a power of two <= 32: the fifth-dimension slices from warp shuffles
      const bool wshfl = g.ls <= 32 && (g.ls & (g.ls - 1)) == 0;
      if (nt != 256) THR_D(1, 1024, false, 1);
      else if (minb == kNoShflCode + 4) THR_D(1, 256, false, 4);  // the slices from memory
      else if (minb == kNoShflCode + 2) THR_D(1, 256, false, 2);
      else if (wshfl && minb == 4) THR_D(1, 256, true, 4);
      else if (wshfl && minb == 3) THR_D(1, 256, true, 3);
      else if (wshfl) THR_D(1, 256, true, 2);
      else if (minb == 4) THR_D(1, 256, false, 4);
      else if (minb == 3) THR_D(1, 256, false, 3);
      else THR_D(1, 256, false, 2);
    } else if (nt != 128) {
      THR_D(0, 1024, false, 1);
    } else if (minb > kNoShflCode && minb < kG2Code) {
      if (minb == kNoShflCode + 8) THR_D(0, 128, false, 8);
      else THR_D(0, 128, false, 6);
    } else if (minb > kG2Code) {
      if constexpr (storage_id<S>() == 0) {
        const int K = (minb - kG2Code) / 10;
        const dim3 gblk(blk.x, K * blk.y, 1);
        const dim3 ggrd((grd.x + K - 1) / K);
        const int np = (int)grd.x;
#define THR_G(D, E, SH, KK, MB)                                                                          \
  launch_k(k_dslash_g2<S, D, E, SH, KK, MB>, ggrd, gblk, 0, st, pdl, out, in, u, g, am, imass, am3, skip, aux, \
           coef, partials, rev, np)
#define THR_GE(D, SH, KK, MB)                \
  do {                                       \
    if (e == 1) THR_G(D, 1, SH, KK, MB);     \
    else if (e == 2) THR_G(D, 2, SH, KK, MB); \
    else if (e == 3) THR_G(D, 3, SH, KK, MB); \
    else THR_G(D, 0, SH, KK, MB);            \
  } while (0)
#define THR_GM(SH, KK, MB)                  \
  do {                                      \
    if (dag) THR_GE(true, SH, KK, MB);      \
    else THR_GE(false, SH, KK, MB);         \
  } while (0)
#define THR_GK(SH)                                          \
  do {                                                      \
    if (minb == kG2Code + 24) THR_GM(SH, 2, 4);             \
    else if (minb == kG2Code + 23) THR_GM(SH, 2, 3);        \
    else if (minb == kG2Code + 42) THR_GM(SH, 4, 2);        \
    else THR_GM(SH, 8, 1);                                  \
  } while (0)
        if (shfl) THR_GK(true);
        else THR_GK(false);
#undef THR_GK
#undef THR_GM
#undef THR_GE
#undef THR_G
      }
    } else if (minb == kSplitCode) {
      if constexpr (storage_id<S>() == 0) {
      const dim3 sblk(blk.x, blk.y, 4);
#define THR_S(D, E, SH)                                                                                  \
  launch_k(k_dslash_split<S, D, E, SH>, grd, sblk, 0, st, pdl, out, in, u, g, am, imass, am3, skip, aux, coef, \
           partials, rev)
#define THR_SE(D, SH)                \
  do {                               \
    if (e == 1) THR_S(D, 1, SH);     \
    else if (e == 2) THR_S(D, 2, SH); \
    else if (e == 3) THR_S(D, 3, SH); \
    else THR_S(D, 0, SH);            \
  } while (0)
      if (shfl) {
        if (dag) THR_SE(true, true);
        else THR_SE(false, true);
      } else {
        if (dag) THR_SE(true, false);
        else THR_SE(false, false);
      }
#undef THR_SE
#undef THR_S
      }
    } else if (shfl) {
      if (minb == 8) THR_D(0, 128, true, 8);
      else if (minb == 7) THR_D(0, 128, true, 7);
      else THR_D(0, 128, true, 6);
    } else {
      if (minb == 8) THR_D(0, 128, false, 8);
      else if (minb == 7) THR_D(0, 128, false, 7);
      else THR_D(0, 128, false, 6);
    }
  };
  const bool tunable = storage_id<S>() < 2 && nt == (kernel == 0 ? 128 : 256);
  // FP64 Shamir, 128-thread blocks: the four-threads-per-site kernel; where a block is
  // whole warps also the two-group blocks
  const bool split_ok = kernel == 0 && storage_id<S>() == 0;
  const bool g2_ok = split_ok && (blk.x * blk.y) % 32 == 0;
  int cand64[kMaxCand] = {8, 7, 6};
  int ncand = 3;
  if (split_ok) {
    cand64[ncand++] = kSplitCode;
    if (g2_ok) {
      cand64[ncand++] = kG2Code + 24;
      cand64[ncand++] = kG2Code + 23;
      cand64[ncand++] = kG2Code + 42;
      cand64[ncand++] = kG2Code + 81;
    }
    if (shfl) {
      cand64[ncand++] = kNoShflCode + 8;
      cand64[ncand++] = kNoShflCode + 6;
    }
  }
  // Wilson with Ls a power of two <= 32: the shuffle kernel's budgets, and the same kernel
  // reading the fifth-dimension slices from memory (the same values and bits)
  int candw[kMaxCand] = {kTuneWilson[0], kTuneWilson[1], kTuneWilson[2]};
  if (kernel == 1 && g.ls <= 32 && (g.ls & (g.ls - 1)) == 0) {
    candw[3] = kNoShflCode + 4;
    candw[4] = kNoShflCode + 2;
    ncand = 5;
  }
  const int* cand = kernel == 0 ? (split_ok ? cand64 : kTuneShamir) : candw;
  int minb = cand[0];
  if (tunable) {
    int dev = 0;
    cudaGetDevice(&dev);
    const TuneKey key{dev, storage_id<S>(), kernel, dag ? 1 : 0, e, g.lx, g.ly, g.lt, g.ls, g.layout};
    minb = may_tune ? tune_pick(key, cand, ncand, st, launch) : tune_lookup(key, cand);
  }
  launch(minb);
#undef THR_D
#undef THR_E
#undef THR_L
  return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
}

template <class S>
int launch_dslash_axpy(const Geom& g, int kernel, bool dag, S* rnew, const S* in, const typename Sto<S>::C* u,
                       float am, int imass, float am3, cudaStream_t st, const int* skip, const S* rold,
                       const double* coef, double* partials, int rev, bool pdl) {
  return launch_dslash_mode<S>(g, kernel, dag, rnew, in, u, am, imass, am3, st, skip, rold, coef, partials, 1, rev,
                               true, pdl);
}

template <class S>
int launch_dslash_accum(const Geom& g, int kernel, bool dag, S* hnew, const S* in, const typename Sto<S>::C* u,
                        float am, int imass, float am3, cudaStream_t st, const int* skip, const S* hold,
                        const double* coef, double* partials, int rev, bool pdl) {
  return launch_dslash_mode<S>(g, kernel, dag, hnew, in, u, am, imass, am3, st, skip, hold, coef, partials, 3, rev,
                               true, pdl);
}

template <class S>
int launch_dslash_norm(const Geom& g, int kernel, bool dag, S* out, const S* in, const typename Sto<S>::C* u,
                       float am, int imass, float am3, cudaStream_t st, const int* skip, double* partials, int rev,
                       bool pdl) {
  return launch_dslash_mode<S>(g, kernel, dag, out, in, u, am, imass, am3, st, skip, nullptr, nullptr, partials, 2,
                               rev, true, pdl);
}

template <class S>
int launch_dslash(const Geom& g, int kernel, bool dag, S* out, const S* in, const typename Sto<S>::C* u, float am,
                  int imass, float am3, cudaStream_t st, const int* skip) {
  return launch_dslash_mode<S>(g, kernel, dag, out, in, u, am, imass, am3, st, skip, nullptr, nullptr, nullptr, 0,
                               0);
}

template <class S>
int launch_dslash_untuned(const Geom& g, int kernel, bool dag, S* out, const S* in, const typename Sto<S>::C* u,
                          float am, int imass, float am3, cudaStream_t st, const int* skip) {
  return launch_dslash_mode<S>(g, kernel, dag, out, in, u, am, imass, am3, st, skip, nullptr, nullptr, nullptr, 0, 0,
                               false);
}

int launch_odslash(const Geom& g, bool dag, double2* out, const double2* in, const double2* u, float am, int imass,
                   float am3, const double* zc, cudaStream_t st, const int* skip) {
  if (g.ls > 1024) return THR_ERR_BADSHAPE;
  if (4ULL * (unsigned long long)g.v5 >= (1ULL << 32)) return THR_ERR_BADSHAPE;  // 32-bit element offsets
  if (imass != 1 && imass != 3) return THR_ERR_UNSUPPORTED;  // measure_OWilson.F90:66-83
  const dim3 blk = stencil_block(g, 1);
  const dim3 grd(stencil_grid(g, 1));
  // register budget (resident 256-thread blocks per SM) tuned per lattice and direction like
  // the other stencils: 4 and 3 win on large lattices, 1 on small ones
#define THR_O(D, MB) k_odslash<D, MB><<<grd, blk, 0, st>>>(out, in, u, g, am, imass, am3, zc, skip)
  auto launch = [&](int mb) {
    if (dag) {
      if (mb == 4) THR_O(true, 4);
      else if (mb == 3) THR_O(true, 3);
      else THR_O(true, 1);
    } else {
      if (mb == 4) THR_O(false, 4);
      else if (mb == 3) THR_O(false, 3);
      else THR_O(false, 1);
    }
  };
#undef THR_O
  int dev = 0;
  cudaGetDevice(&dev);
  const int mb = tune_pick(TuneKey{dev, 0, 2, dag ? 1 : 0, 0, g.lx, g.ly, g.lt, g.ls, g.layout}, kTuneOverlap, 3, st,
                           launch);
  launch(mb);
  return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
}

// The persistent batch stencil's grid (resident blocks per SM) is tuned like the register
// budgets: work blocks, not CTAs, own the partial sums, so every grid gives the same bits.
constexpr int kTuneBatchGrid[3] = {8, 4, 16};  // CTAs per SM

template <class S>
int launch_dslash_batch(const BatchTable& b, int kernel, bool dag, S* out, const S* in, const typename Sto<S>::C* u,
                        float am, int imass, float am3, cudaStream_t st, const int* skip, const S* aux,
                        double* partials, int grid) {
  if (kernel == 1 && imass != 1 && imass != 3) return THR_ERR_UNSUPPORTED;
  const bool epi = aux != nullptr;
  auto launch = [&](int per_sm) {
    const int g = grid > 0 ? grid : std::min(b.total_blocks, device_sms() * per_sm);
#define THR_L(K, D, E)                                                                                          \
  k_dslash_batch<S, K, D, E><<<g, 256, 0, st>>>(out, in, u, b.dev, b.nent, b.total_blocks, am, imass, am3, skip, \
                                                aux, partials, nullptr, nullptr, 0)
    if (kernel == 1) {
      if (dag) { if (epi) THR_L(1, true, 1); else THR_L(1, true, 0); }
      else { if (epi) THR_L(1, false, 1); else THR_L(1, false, 0); }
    } else {
      if (dag) { if (epi) THR_L(0, true, 1); else THR_L(0, true, 0); }
      else { if (epi) THR_L(0, false, 1); else THR_L(0, false, 0); }
    }
#undef THR_L
  };
  int per_sm = kTuneBatchGrid[0];
  if (grid <= 0 && b.total_blocks > device_sms() * kTuneBatchGrid[1]) {
    int dev = 0;
    cudaGetDevice(&dev);
    // key: the batch kernel family (10 + kernel), its size (total work blocks, entries)
    per_sm = tune_pick(TuneKey{dev, storage_id<S>(), 10 + kernel, dag ? 1 : 0, epi ? 1 : 0, b.total_blocks, b.nent, 0,
                               0, 0},
                       kTuneBatchGrid, 3, st, launch);
  }
  launch(per_sm);
  return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
}

template <class S>
int launch_dslash_batch_fused(const BatchTable& b, int kernel, bool dag, int epi, S* out, const S* in,
                              const typename Sto<S>::C* u, float am, int imass, float am3, cudaStream_t st,
                              const int* skip, typename Sto<S>::C* rv, const double* coef, int coef_stride,
                              double* partials, int grid) {
  if (kernel == 1 && imass != 1 && imass != 3) return THR_ERR_UNSUPPORTED;
  if (epi != 2 && epi != 4) return THR_ERR_BADARG;
  auto launch = [&](int per_sm) {
    const int g = grid > 0 ? grid : std::min(b.total_blocks, device_sms() * per_sm);
#define THR_L(K, D, E)                                                                                          \
  k_dslash_batch<S, K, D, E><<<g, 256, 0, st>>>(out, in, u, b.dev, b.nent, b.total_blocks, am, imass, am3, skip, \
                                                nullptr, partials, rv, coef, coef_stride)
    if (kernel == 1) {
      if (dag) { if (epi == 4) THR_L(1, true, 4); else THR_L(1, true, 2); }
      else { if (epi == 4) THR_L(1, false, 4); else THR_L(1, false, 2); }
    } else {
      if (dag) { if (epi == 4) THR_L(0, true, 4); else THR_L(0, true, 2); }
      else { if (epi == 4) THR_L(0, false, 4); else THR_L(0, false, 2); }
    }
#undef THR_L
  };
  int per_sm = kTuneBatchGrid[0];
  if (grid <= 0 && b.total_blocks > device_sms() * kTuneBatchGrid[1]) {
    int dev = 0;
    cudaGetDevice(&dev);
    // epi 4 updates rv in place, so it is never launched for timing: it takes the grid
    // tuned for the same batch's M with |M p|^2 (epi 2)
    const TuneKey k2{dev, storage_id<S>(), 10 + kernel, 0, 2, b.total_blocks, b.nent, 0, 0, 0};
    per_sm = epi == 4 ? tune_lookup(k2, kTuneBatchGrid)
                      : tune_pick(TuneKey{dev, storage_id<S>(), 10 + kernel, dag ? 1 : 0, 2, b.total_blocks, b.nent,
                                          0, 0, 0},
                                  kTuneBatchGrid, 3, st, launch);
  }
  launch(per_sm);
  return cudaPeekAtLastError() == cudaSuccess ? THR_OK : THR_ERR_CUDA;
}

#define THR_INST(S, L)                                                                                            \
  template int launch_dslash<S>(const Geom&, int, bool, S*, const S*, const L*, float, int, float, cudaStream_t,   \
                                const int*);                                                                      \
  template int launch_dslash_untuned<S>(const Geom&, int, bool, S*, const S*, const L*, float, int, float,        \
                                        cudaStream_t, const int*);                                                \
  template int launch_dslash_axpy<S>(const Geom&, int, bool, S*, const S*, const L*, float, int, float,           \
                                     cudaStream_t, const int*, const S*, const double*, double*, int, bool);      \
  template int launch_dslash_norm<S>(const Geom&, int, bool, S*, const S*, const L*, float, int, float,           \
                                     cudaStream_t, const int*, double*, int, bool);                               \
  template int launch_dslash_accum<S>(const Geom&, int, bool, S*, const S*, const L*, float, int, float,          \
                                      cudaStream_t, const int*, const S*, const double*, double*, int, bool);     \
  template int launch_dslash_batch<S>(const BatchTable&, int, bool, S*, const S*, const L*, float, int, float,    \
                                      cudaStream_t, const int*, const S*, double*, int);                          \
  template int launch_dslash_batch_fused<S>(const BatchTable&, int, bool, int, S*, const S*, const L*, float, int, \
                                            float, cudaStream_t, const int*, L*, const double*, int, double*, int);
THR_INST(double2, double2)
THR_INST(float2, float2)
THR_INST(__nv_bfloat162, float2)
THR_INST(__half2, float2)
#undef THR_INST

}  // namespace thr

// Blocks of the staged-tile stencil whose copies did not arrive in time, on the context's device
extern "C" int thr_stencil_timeouts(thr_ctx* c, unsigned long long* count) {
  if (!c || !count) return THR_ERR_BADARG;
  cudaSetDevice(c->dev);
  return cudaMemcpyFromSymbol(count, thr::g_stencil_timeouts, sizeof(unsigned long long)) == cudaSuccess
             ? THR_OK
             : THR_ERR_CUDA;
}

// The autotuner's choices so far, one line each:
//   <storage> <shamir|wilson|overlap> <M|Mdag> epi=<e> <lx>x<ly>x<lt> Ls=<ls> layout=<l> dev=<d> minb=<pick> us=<per candidate>
extern "C" int thr_tune_report(char* buf, int len) {
  using namespace thr;
  if (!buf || len < 1) return THR_ERR_BADARG;
  std::string r;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    for (const auto& kv : g_tune) {
      const TuneKey& k = kv.first;
      char line[256];
      const char* sto = k.sid == 0 ? "fp64" : k.sid == 1 ? "fp32" : "bf16";
      int w;
      if (k.ker >= 10)  // persistent batch stencil: lx = its work blocks, ly = entries
        w = std::snprintf(line, sizeof(line), "%s batch-%s %s epi=%d blocks=%d entries=%d dev=%d ctas_per_sm=%d us=",
                          sto, k.ker == 11 ? "wilson" : "shamir", k.dag ? "Mdag" : "M", k.epi, k.lx, k.ly, k.dev,
                          kv.second.pick);
      else
        w = std::snprintf(line, sizeof(line), "%s %s %s epi=%d %dx%dx%d Ls=%d layout=%d dev=%d minb=%d us=", sto,
                          k.ker == 2 ? "overlap" : k.ker ? "wilson" : "shamir", k.dag ? "Mdag" : "M", k.epi, k.lx,
                          k.ly, k.lt, k.ls, k.layout, k.dev, kv.second.pick);
      for (int c = 0; c < kv.second.ncand && w > 0 && w < (int)sizeof(line); c++)
        w += std::snprintf(line + w, sizeof(line) - w, c ? "/%.2f" : "%.2f", kv.second.us[c]);
      r += line;
      r += "\n";
    }
  }
  std::snprintf(buf, (size_t)len, "%s", r.c_str());
  return THR_OK;
}
