// dslash_site.cuh -- the per-site arithmetic of the domain-wall operator and the
// block body of the one-thread-per-5D-site stencil, shared by the stencil kernels
// (dslash.cu) and the persistent solver kernel of the batched multishift (msp.cu),
// so both run the same instructions per site and give the same bits.
#pragma once
#include "ctx.h"
#include "thr_common.cuh"

namespace thr {


// Spinor loads: COH false reads through the read-only path (__ldg), for fields no
// thread writes during the launch; COH true through L2 (__ldcg), for the persistent
// solver kernel, whose blocks read fields other blocks wrote earlier in the same launch.
template <class S, bool COH>
__device__ __forceinline__ typename Sto<S>::C sto_ld(const S* p, size_t i) {
  if constexpr (COH) return Sto<S>::ldcg(p, i);
  else return Sto<S>::ld(p, i);
}

template <class S, bool COH = false>
struct SpinorView {
  const S* p;
  Geom g;
  __device__ __forceinline__ typename Sto<S>::C operator()(int s, int site, int d) const {
    return sto_ld<S, COH>(p, sidx32(g, s, site, d));
  }
};

// Re(conj(aux_i) v) in the working precision, accumulated in FP64 (for FP32
// storage the term is an FP32 value summed in FP64, as reduce_real_dp5d does)
template <class S>
__device__ __forceinline__ double epi_redot(const S* aux, size_t i, typename Sto<S>::C v) {
  using R = typename Sto<S>::R;
  const typename Sto<S>::C a = Sto<S>::ld(aux, i);
  const R t = a.x * v.x + a.y * v.y;
  return (double)t;
}

// |v|^2 in the working precision, accumulated in FP64
template <class S>
__device__ __forceinline__ double epi_norm(typename Sto<S>::C v) {
  using R = typename Sto<S>::R;
  const R t = v.x * v.x + v.y * v.y;
  return (double)t;
}

// ---------------------------------------------------------------- Shamir
// One hop of the 3D Wilson-Dirac term, spin-projected.  The reference adds
// -1/2 [T(d) -+ 2gamma(mu,d) T(gin)] with T = W R(neighbour) for each d
// (dirac.F90:49-76, :464-491).  2gamma(mu,.) is a Hermitian unitary permutation
// (entries +-1, +-i) pairing each upper spin with a lower one, so
//   h(d) = R(d) -+ 2gamma(mu,d) R(gin)   for the upper spins d = 0, 1
// carries the whole hop: W h(d) goes to spin d and -+2gamma(mu,gin) W h(d) to
// spin gin.  Two complex multiplies per neighbour instead of four; the result
// differs from the unprojected sum by rounding only.
// The hop in two parts: hop_products forms W h(d) for d = 0, 1 from the neighbour's
// spinor, hop_accumulate adds them into the site's sums (the four-threads-per-site
// stencil runs the two parts in different threads).
template <class C>
__device__ __forceinline__ void hop_products(int mu, bool plus, C W, const C* r, C* wh) {
#pragma unroll
  for (int d = 0; d < 2; d++) {
    const GammaEntry ge = gamma_entry(mu, d);
    const C gr = gp(ge, r[ge.gin]);
    wh[d] = cmul(W, plus ? r[d] - gr : r[d] + gr);
  }
}
template <class C, class R>
__device__ __forceinline__ void hop_accumulate(int mu, bool plus, const C* wh, C* acc) {
#pragma unroll
  for (int d = 0; d < 2; d++) {
    const int gi = gamma_entry(mu, d).gin;
    acc[d] = acc[d] - R(0.5) * wh[d];
    const C gw = gp(gamma_entry(mu, gi), wh[d]);
    acc[gi] = plus ? acc[gi] + R(0.5) * gw : acc[gi] - R(0.5) * gw;
  }
}
// the two parts in one pass, d by d (the one-thread-per-site kernels)
template <class C, class R>
__device__ __forceinline__ void hop_projected(int mu, bool plus, C W, const C* r, C* acc) {
#pragma unroll
  for (int d = 0; d < 2; d++) {
    const GammaEntry ge = gamma_entry(mu, d);
    const int gi = ge.gin;
    const C gr = gp(ge, r[gi]);
    const C wh = cmul(W, plus ? r[d] - gr : r[d] + gr);
    acc[d] = acc[d] - R(0.5) * wh;
    const C gw = gp(gamma_entry(mu, gi), wh);
    acc[gi] = plus ? acc[gi] + R(0.5) * gw : acc[gi] - R(0.5) * gw;
  }
}

// The site-local terms of the Shamir operator (diagonal, fifth-dimension hop, wall mass
// term) into acc.  SHFL: the fifth-dimension neighbours and wall values come from the
// lanes of the same site (blockDim.x = Ls a power of two <= 32, so a site's Ls threads
// are one aligned segment of a warp); every lane must call this.
template <class S, bool DAG, bool SHFL, bool COH = false>
__device__ __forceinline__ void shamir_local(const S* __restrict__ in, const Geom& g, int s, int site, float am,
                                             int imass, float am3, typename Sto<S>::C* acc) {
  using R = typename Sto<S>::R;
  using C = typename Sto<S>::C;
  SpinorView<S, COH> Rv{in, g};
  const int Ls = g.ls;
  const R diag = (R)((3.0f - am3) + 1.0f);  // dirac.F90:45, default real
  C rc[4];
#pragma unroll
  for (int d = 0; d < 4; d++) {
    rc[d] = Rv(s, site, d);
    acc[d] = diag * rc[d];
  }
  // fifth-dimension hop (np_third == 1), dirac.F90:80-87 (M), :317-324 (M^dagger):
  // spins A take R(s+1), spins B take R(s-1); A = (2,3) for M, (0,1) for M^dagger
  const int a0 = DAG ? 0 : 2, b0 = DAG ? 2 : 0;
  C nxt[2], prv[2], w0[2], wl[2];
  if (SHFL) {
    const unsigned full = 0xffffffffu;
#pragma unroll
    for (int k = 0; k < 2; k++) {
      nxt[k] = mk(__shfl_down_sync(full, rc[a0 + k].x, 1, Ls), __shfl_down_sync(full, rc[a0 + k].y, 1, Ls));
      prv[k] = mk(__shfl_up_sync(full, rc[b0 + k].x, 1, Ls), __shfl_up_sync(full, rc[b0 + k].y, 1, Ls));
      w0[k] = mk(__shfl_sync(full, rc[a0 + k].x, 0, Ls), __shfl_sync(full, rc[a0 + k].y, 0, Ls));
      wl[k] = mk(__shfl_sync(full, rc[b0 + k].x, Ls - 1, Ls), __shfl_sync(full, rc[b0 + k].y, Ls - 1, Ls));
    }
  }
#pragma unroll
  for (int k = 0; k < 2; k++) {
    if (s < Ls - 1) acc[a0 + k] = acc[a0 + k] - (SHFL ? nxt[k] : Rv(s + 1, site, a0 + k));
    if (s > 0) acc[b0 + k] = acc[b0 + k] - (SHFL ? prv[k] : Rv(s - 1, site, b0 + k));
  }
  // wall mass term: dirac.F90:119-176 (M), :356-402 (M^dagger).  imass 1, 3 couple
  // R(1) into s = Ls (spins A) and R(Ls) into s = 1 (spins B); imass 5 mixes the
  // chiralities at the same s.  Written as acc += c * v with one coefficient per
  // wall: imass 1: am; imass 3: +i am (A), -i am (B); imass 5: +-i am (M / M^dagger).
  const R a = (R)am;
  const bool five = imass == 5;
  const C cA = imass == 1 ? mk(a, R(0)) : mk(R(0), (five && DAG) ? -a : a);
  const C cB = imass == 1 ? mk(a, R(0)) : mk(R(0), five ? (DAG ? -a : a) : -a);
#pragma unroll
  for (int k = 0; k < 2; k++) {
    if (s == Ls - 1)
      acc[a0 + k] = acc[a0 + k] + cmul(cA, five ? rc[b0 + k] : (SHFL ? w0[k] : Rv(0, site, a0 + k)));
    if (s == 0)
      acc[b0 + k] = acc[b0 + k] + cmul(cB, five ? rc[a0 + k] : (SHFL ? wl[k] : Rv(Ls - 1, site, b0 + k)));
  }
}

// The whole Shamir operator at one 5D site: the local terms, then the Wilson and Dirac
// hopping terms, forward (U R(x+mu)) then backward (conj U(x-mu) R(x-mu)) per
// direction; +gamma forward and -gamma backward in M, the opposite in M^dagger.  The
// reference adds them before (M) or after (M^dagger) the fifth-dimension and mass
// terms; the order only affects rounding.
template <class S, bool DAG, bool SHFL, bool COH = false>
__device__ __forceinline__ void shamir_site(const S* __restrict__ in, const typename Sto<S>::C* __restrict__ u,
                                            const Geom& g, int s, int site, float am, int imass, float am3,
                                            typename Sto<S>::C* acc) {
  using R = typename Sto<S>::R;
  using C = typename Sto<S>::C;
  int x, y, t;
  site_coords(g, site, x, y, t);
  const Nbr nb = neighbours(g, site, x, y, t);
  SpinorView<S, COH> Rv{in, g};
  shamir_local<S, DAG, SHFL, COH>(in, g, s, site, am, imass, am3, acc);
#pragma unroll
  for (int mu = 0; mu < 3; mu++) {
#pragma unroll
    for (int dir = 0; dir < 2; dir++) {
      const int ns = dir == 0 ? nb.f[mu] : nb.b[mu];
      const C W = dir == 0 ? __ldg(u + (size_t)mu * g.v3 + site) : cconj(__ldg(u + (size_t)mu * g.v3 + nb.b[mu]));
      C r[4];
#pragma unroll
      for (int d = 0; d < 4; d++) r[d] = Rv(s, ns, d);
      hop_projected<C, R>(mu, (dir == 0) != DAG, W, r, acc);
    }
  }
}

// ---------------------------------------------------------------- Wilson
// a complex value from lane `src` of this lane's Ls-wide segment (every lane calls it)
template <class C>
__device__ __forceinline__ C seg_shfl(C v, int src, int Ls) {
  return mk(__shfl_sync(0xffffffffu, v.x, src, Ls), __shfl_sync(0xffffffffu, v.y, src, Ls));
}

// Q(s) components for the forward operator at (s, site).  SHFL: the slices s-1, s+1 and
// the walls' R(Ls), R(1) come from the lanes of the same site (blockDim.x = Ls a power of
// two <= 32; every lane must call this): the same values, one load per spin instead of three.
template <class S, bool COH, bool SHFL = false>
__device__ __forceinline__ void wilson_q(const SpinorView<S, COH>& Rv, int s, int site, int Ls,
                                         typename Sto<S>::C c1, typename Sto<S>::C c2,
                                         typename Sto<S>::C* q) {
  using C = typename Sto<S>::C;
  C r[4];
#pragma unroll
  for (int d = 0; d < 4; d++) r[d] = Rv(s, site, d);
  if (SHFL) {
#pragma unroll
    for (int d = 0; d < 2; d++) {
      const C prv = seg_shfl(r[d], s > 0 ? s - 1 : Ls - 1, Ls);
      q[d] = (s > 0) ? r[d] + prv : r[d] + cmul(c1, prv);
    }
#pragma unroll
    for (int d = 2; d < 4; d++) {
      const C nxt = seg_shfl(r[d], s < Ls - 1 ? s + 1 : 0, Ls);
      q[d] = (s < Ls - 1) ? r[d] + nxt : r[d] + cmul(c2, nxt);
    }
    return;
  }
  // P+ (spins 0,1) from s-1, wall: c1 * R(Ls)
#pragma unroll
  for (int d = 0; d < 2; d++) q[d] = (s > 0) ? r[d] + Rv(s - 1, site, d) : r[d] + cmul(c1, Rv(Ls - 1, site, d));
  // P- (spins 2,3) from s+1, wall: c2 * R(1)
#pragma unroll
  for (int d = 2; d < 4; d++) q[d] = (s < Ls - 1) ? r[d] + Rv(s + 1, site, d) : r[d] + cmul(c2, Rv(0, site, d));
}

template <class S, bool DAG, bool COH = false, bool SHFL = false>
__device__ __forceinline__ void wilson_site(const S* __restrict__ in, const typename Sto<S>::C* __restrict__ u,
                                            const Geom& g, int s, int site, float am, int imass, float am3,
                                            typename Sto<S>::C* res) {
  using R = typename Sto<S>::R;
  using C = typename Sto<S>::C;
  int x, y, t;
  site_coords(g, site, x, y, t);
  const Nbr nb = neighbours(g, site, x, y, t);
  SpinorView<S, COH> Rv{in, g};
  const int Ls = g.ls;
  const R a = (R)am;
  const R dgw = (R)(3.0f + (-am3));  // DWilson(…, -am3) diagonal: dirac.F90:191, :505
  if (!DAG) {
    // c1 = -am | -i am  (dirac.F90:274-278),  c2 = -am | +i am  (dirac.F90:287-291)
    const C c1 = imass == 1 ? mk(-a, R(0)) : mk(R(0), -a);
    const C c2 = imass == 1 ? mk(-a, R(0)) : mk(R(0), a);
    C q[4];
    wilson_q<S, COH, SHFL>(Rv, s, site, Ls, c1, c2, q);
#pragma unroll
    for (int d = 0; d < 4; d++) res[d] = (dgw - R(1)) * q[d] + R(2) * Rv(s, site, d);
    // D_W hops of Q (dirac.F90:197-217), spin-projected as in the Shamir kernel
#pragma unroll
    for (int mu = 0; mu < 3; mu++) {
      const C U = __ldg(u + (size_t)mu * g.v3 + site);
      const C Ub = cconj(__ldg(u + (size_t)mu * g.v3 + nb.b[mu]));
      C q[4];
      wilson_q<S, COH, SHFL>(Rv, s, nb.f[mu], Ls, c1, c2, q);
      hop_projected<C, R>(mu, true, U, q, res);
      wilson_q<S, COH, SHFL>(Rv, s, nb.b[mu], Ls, c1, c2, q);
      hop_projected<C, R>(mu, false, Ub, q, res);
    }
  } else {
    // z = -am | -i am (upper right, dirac.F90:602-606); z' = -am | +i am (lower left, :615-619)
    const C z = imass == 1 ? mk(-a, R(0)) : mk(R(0), -a);
    const C zp = imass == 1 ? mk(-a, R(0)) : mk(R(0), a);
    // half 0: output spins 0,1 use Qp = R(s) + R(s+1) | z' R(1); half 1: spins 2,3 use Qm = R(s) + R(s-1) | z R(Ls).
    // One pass over the neighbours serves both halves: R(s) and the two partner slices are loaded
    // once per site (each output element gets the same operations in the same order as half by half)
    const bool in0 = s < Ls - 1, in1 = s > 0;
    const int sp0 = in0 ? s + 1 : 0, sp1 = in1 ? s - 1 : Ls - 1;
    auto qpair = [&](int st, C* q0, C* q1) {
#pragma unroll
      for (int d = 0; d < 4; d++) {
        const C r = Rv(s, st, d);
        const C a0 = SHFL ? seg_shfl(r, sp0, Ls) : Rv(sp0, st, d);
        const C a1 = SHFL ? seg_shfl(r, sp1, Ls) : Rv(sp1, st, d);
        q0[d] = in0 ? r + a0 : r + cmul(zp, a0);
        q1[d] = in1 ? r + a1 : r + cmul(z, a1);
      }
    };
    {
      C q0[4], q1[4];
      qpair(site, q0, q1);
#pragma unroll
      for (int k = 0; k < 2; k++) {
        res[k] = (dgw - R(1)) * q0[k] + R(2) * Rv(s, site, k);
        res[2 + k] = (dgw - R(1)) * q1[2 + k] + R(2) * Rv(s, site, 2 + k);
      }
    }
    // D_W^dagger hops (dirac.F90:511-531): -1/2 W [q(d) +- 2gamma(mu,d) q(gin)], each half's
    // output spins from its own Q
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

template <class S, int KER, bool DAG, bool SHFL = false, bool COH = false>
__device__ __forceinline__ void apply_site(const S* in, const typename Sto<S>::C* u, const Geom& g, int s, int site,
                                           float am, int imass, float am3, typename Sto<S>::C* acc) {
  if (KER == 0) shamir_site<S, DAG, SHFL, COH>(in, u, g, s, site, am, imass, am3, acc);
  else wilson_site<S, DAG, COH, SHFL>(in, u, g, s, site, am, imass, am3, acc);
}

// One block's sites of the stencil with its epilogue (blockDim = (Ls, sites per
// block), NT threads at most; the block's sites are bid * blockDim.y + threadIdx.y).
// Epilogues (EPI): 0 store out = M in; 2 also one FP64 partial of |out|^2 into
// partials[bid]; 1 out = aux + om * (M in), with M in never stored, and a partial of
// |out|^2; 3 out = M in + om * aux with a partial of |out|^2.  The partial goes through
// shared memory and the block's first warp in a fixed order.  A caller that runs
// another block body right after this one must __syncthreads() in between (the
// partial's shared array is reused).  COH: spinor loads through L2 (see sto_ld).
// The persistent multishift kernel runs the same pieces (block_sites, epi_element,
// block_partial_sum) with work of its own between the stencil and its epilogue.

// the epilogue of one output element i from the stencil's value v
template <class S, int EPI, bool COH>
__device__ __forceinline__ void epi_element(S* __restrict__ out, const S* __restrict__ aux, typename Sto<S>::R om,
                                            unsigned i, typename Sto<S>::C v, double& racc) {
  using C = typename Sto<S>::C;
  if (EPI == 1) {
    const C rn = sto_ld<S, COH>(aux, i) + om * v;  // r = r + omega*s (multishift_module.F90:137)
    Sto<S>::st(out, i, rn);
    racc += epi_norm<S>(rn);
  } else if (EPI == 3) {
    const C hn = v + om * sto_ld<S, COH>(aux, i);  // h = M r + gamma h (= M p by linearity)
    Sto<S>::st(out, i, hn);
    racc += epi_norm<S>(hn);
  } else {
    Sto<S>::st(out, i, v);
    if (EPI == 2) racc += epi_norm<S>(v);
  }
}

// one FP64 partial per block in a fixed order.  Blocks of Ls x sites need not be
// whole warps (Ls = 12: 120 threads), so the values go through shared memory and
// the first warp -- always complete: every configuration has >= 32 threads -- sums them.
template <int NT>
__device__ __forceinline__ void block_partial_sum(double racc, double* __restrict__ partials, int bid) {
  __shared__ double red[NT];
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

template <class S, int KER, bool DAG, int EPI, int NT, bool SHFL, bool COH = false>
__device__ __forceinline__ void dslash_block(S* __restrict__ out, const S* __restrict__ in,
                                             const typename Sto<S>::C* __restrict__ u, const Geom& g, float am,
                                             int imass, float am3, const S* __restrict__ aux,
                                             typename Sto<S>::R om, int bid, double* __restrict__ partials) {
  using C = typename Sto<S>::C;
  const int s = threadIdx.x;
  double racc = 0.0;
  const int site = bid * blockDim.y + threadIdx.y;
  const bool live = site < g.v3;
  if (SHFL || live) {  // with SHFL every lane takes part (the last block's spare rows on a clamped site)
    const int st = live ? site : g.v3 - 1;
    C acc[4];
    apply_site<S, KER, DAG, SHFL, COH>(in, u, g, s, st, am, imass, am3, acc);
    if (live) {
#pragma unroll
      for (int d = 0; d < 4; d++) epi_element<S, EPI, COH>(out, aux, om, sidx32(g, s, site, d), acc[d], racc);
    }
  }
  if (EPI != 0) block_partial_sum<NT>(racc, partials, bid);
}

// the stencil part of dslash_block alone: the thread's M in (acc); spare rows compute a
// clamped site (SHFL) or nothing
template <class S, int KER, bool DAG, bool SHFL, bool COH = false>
__device__ __forceinline__ void block_sites(const S* __restrict__ in, const typename Sto<S>::C* __restrict__ u,
                                            const Geom& g, float am, int imass, float am3, int bid,
                                            typename Sto<S>::C* acc) {
  const int s = threadIdx.x;
  const int site = bid * blockDim.y + threadIdx.y;
  const bool live = site < g.v3;
  if (SHFL || live) {
    const int st = live ? site : g.v3 - 1;
    apply_site<S, KER, DAG, SHFL, COH>(in, u, g, s, st, am, imass, am3, acc);
  }
}

}  // namespace thr
