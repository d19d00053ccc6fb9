/*
 * thirring_oracle.c -- CPU restatement of the thirring-rhmc fermion hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker and timed CPU baseline for the
 * CUDA library.  Nothing in the product library calls into this file.
 *
 * Each function follows the cited Fortran routine of the reference
 * (j-ostmeyer/thirring-rhmc) statement by statement, keeping its mixed
 * single/double precision: am, am3, res, diag, tzi_real, theta and pp are
 * single precision exactly where the Fortran declares them `real`.
 * Built with -ffp-contract=off so that every product and sum is rounded as
 * written.  OpenMP parallelises the site loops; per-element operation order
 * is unchanged by it.
 */
#include "thirring_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* indexing                                                                  */
/* ------------------------------------------------------------------------ */
#define LS2 ((size_t)(L->ls + 2))
#define LX2 ((size_t)(L->lx + 2))
#define LY2 ((size_t)(L->ly + 2))
#define LT2 ((size_t)(L->lt + 2))

/* spinor (0:Ls+1,0:Lx+1,0:Ly+1,0:Lt+1,4); d is 0-based */
#define I5(s, x, y, t, d) ((size_t)(s) + LS2 * ((size_t)(x) + LX2 * ((size_t)(y) + LY2 * ((size_t)(t) + LT2 * (size_t)(d)))))
/* link-like (0:Lx+1,0:Ly+1,0:Lt+1,n); c is 0-based */
#define I4(x, y, t, c) ((size_t)(x) + LX2 * ((size_t)(y) + LY2 * ((size_t)(t) + LT2 * (size_t)(c))))
/* (Lx,Ly,Lt,3) with 1-based x,y,t and 0-based mu */
#define I3(x, y, t, c) ((size_t)((x)-1) + (size_t)L->lx * ((size_t)((y)-1) + (size_t)L->ly * ((size_t)((t)-1) + (size_t)L->lt * (size_t)(c))))
/* (Ls,Lx,Ly,Lt,4,ndiag) with 1-based s..t, 0-based d and k */
#define IO(s, x, y, t, d, k) ((size_t)((s)-1) + (size_t)L->ls * ((size_t)((x)-1) + (size_t)L->lx * ((size_t)((y)-1) + (size_t)L->ly * ((size_t)((t)-1) + (size_t)L->lt * ((size_t)(d) + 4 * (size_t)(k))))))

size_t orc_n5(const orc_lat *L) { return LS2 * LX2 * LY2 * LT2 * 4; }
size_t orc_n4(const orc_lat *L) { return LX2 * LY2 * LT2; }
static size_t nout(const orc_lat *L) { return (size_t)L->ls * L->lx * L->ly * L->lt * 4; }

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void orc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* ------------------------------------------------------------------------ */
/* complex arithmetic, Fortran semantics                                     */
/* ------------------------------------------------------------------------ */
static inline orc_zd zd(double r, double i) { orc_zd z = {r, i}; return z; }
static inline orc_zd zadd(orc_zd a, orc_zd b) { return zd(a.re + b.re, a.im + b.im); }
static inline orc_zd zsub(orc_zd a, orc_zd b) { return zd(a.re - b.re, a.im - b.im); }
static inline orc_zd zmul(orc_zd a, orc_zd b) { return zd(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static inline orc_zd zscal(double s, orc_zd a) { return zd(s * a.re, s * a.im); }
static inline orc_zd zconj(orc_zd a) { return zd(a.re, -a.im); }

static inline orc_zf zf(float r, float i) { orc_zf z = {r, i}; return z; }
static inline orc_zf fadd(orc_zf a, orc_zf b) { return zf(a.re + b.re, a.im + b.im); }
static inline orc_zf fsub(orc_zf a, orc_zf b) { return zf(a.re - b.re, a.im - b.im); }
static inline orc_zf fmulz(orc_zf a, orc_zf b) { return zf(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static inline orc_zf fscal(float s, orc_zf a) { return zf(s * a.re, s * a.im); }
static inline orc_zf fconj(orc_zf a) { return zf(a.re, -a.im); }

/* ------------------------------------------------------------------------ */
/* gamma matrices: gammamatrices.F90:17-132                                  */
/* ------------------------------------------------------------------------ */
/* value codes: 1 = +1, -1 = -1, 2 = +i, -2 = -i (before the akappa scaling) */
static const int GAM_CODE[6][4] = {{-2, -2, 2, 2}, {-1, 1, 1, -1}, {-2, 2, 2, -2},
                                   {1, 1, -1, -1}, {-1, -1, -1, -1}, {-1, -1, 1, 1}};
static const int GAM_IN[6][4] = {{3, 2, 1, 0}, {3, 2, 1, 0}, {2, 3, 0, 1},
                                 {0, 1, 2, 3}, {2, 3, 0, 1}, {2, 3, 0, 1}};
static const double AKAPPA = 0.5;
static const float AKAPPAF = 0.5f;

static orc_zd gamval(int mu, int d) {
  int c = GAM_CODE[mu][d];
  orc_zd v = (c == 1) ? zd(1, 0) : (c == -1) ? zd(-1, 0) : (c == 2) ? zd(0, 1) : zd(0, -1);
  return zd(v.re * AKAPPA, v.im * AKAPPA); /* gammamatrices.F90:128 */
}
static orc_zf gamvalf(int mu, int d) {
  int c = GAM_CODE[mu][d];
  orc_zf v = (c == 1) ? zf(1, 0) : (c == -1) ? zf(-1, 0) : (c == 2) ? zf(0, 1) : zf(0, -1);
  return zf(v.re * AKAPPAF, v.im * AKAPPAF); /* gammamatrices.F90:129 */
}
void orc_gammas(int mu, int d, orc_zd *val, int *gin) {
  if (val) *val = gamval(mu, d);
  if (gin) *gin = GAM_IN[mu][d];
}

/* ------------------------------------------------------------------------ */
/* halo updates (periodic, faces only as the MPI subarray types do)          */
/* ------------------------------------------------------------------------ */
#define HALO5_BODY(T, a)                                                                 \
  for (int d = 0; d < 4; d++) {                                                          \
    for (int t = 1; t <= L->lt; t++)                                                     \
      for (int y = 1; y <= L->ly; y++)                                                   \
        for (int s = 1; s <= L->ls; s++) {                                               \
          a[I5(s, 0, y, t, d)] = a[I5(s, L->lx, y, t, d)];                               \
          a[I5(s, L->lx + 1, y, t, d)] = a[I5(s, 1, y, t, d)];                           \
        }                                                                                \
    for (int t = 1; t <= L->lt; t++)                                                     \
      for (int x = 1; x <= L->lx; x++)                                                   \
        for (int s = 1; s <= L->ls; s++) {                                               \
          a[I5(s, x, 0, t, d)] = a[I5(s, x, L->ly, t, d)];                               \
          a[I5(s, x, L->ly + 1, t, d)] = a[I5(s, x, 1, t, d)];                           \
        }                                                                                \
    for (int y = 1; y <= L->ly; y++)                                                     \
      for (int x = 1; x <= L->lx; x++)                                                   \
        for (int s = 1; s <= L->ls; s++) {                                               \
          a[I5(s, x, y, 0, d)] = a[I5(s, x, y, L->lt, d)];                               \
          a[I5(s, x, y, L->lt + 1, d)] = a[I5(s, x, y, 1, d)];                           \
        }                                                                                \
    for (int t = 1; t <= L->lt; t++)                                                     \
      for (int y = 1; y <= L->ly; y++)                                                   \
        for (int x = 1; x <= L->lx; x++) {                                               \
          a[I5(0, x, y, t, d)] = a[I5(L->ls, x, y, t, d)];                               \
          a[I5(L->ls + 1, x, y, t, d)] = a[I5(1, x, y, t, d)];                           \
        }                                                                                \
  }

void orc_update_halo_5(const orc_lat *L, orc_zd *a) { HALO5_BODY(orc_zd, a) }
void orc_update_halo_5_sp(const orc_lat *L, orc_zf *a) { HALO5_BODY(orc_zf, a) }

#define HALO4_BODY(a)                                                                    \
  for (int c = 0; c < n; c++) {                                                          \
    for (int t = 1; t <= L->lt; t++)                                                     \
      for (int y = 1; y <= L->ly; y++) {                                                 \
        a[I4(0, y, t, c)] = a[I4(L->lx, y, t, c)];                                       \
        a[I4(L->lx + 1, y, t, c)] = a[I4(1, y, t, c)];                                   \
      }                                                                                  \
    for (int t = 1; t <= L->lt; t++)                                                     \
      for (int x = 1; x <= L->lx; x++) {                                                 \
        a[I4(x, 0, t, c)] = a[I4(x, L->ly, t, c)];                                       \
        a[I4(x, L->ly + 1, t, c)] = a[I4(x, 1, t, c)];                                   \
      }                                                                                  \
    for (int y = 1; y <= L->ly; y++)                                                     \
      for (int x = 1; x <= L->lx; x++) {                                                 \
        a[I4(x, y, 0, c)] = a[I4(x, y, L->lt, c)];                                       \
        a[I4(x, y, L->lt + 1, c)] = a[I4(x, y, 1, c)];                                   \
      }                                                                                  \
  }
void orc_update_halo_4(const orc_lat *L, int n, orc_zd *a) { HALO4_BODY(a) }
void orc_update_halo_4_real(const orc_lat *L, int n, float *a) { HALO4_BODY(a) }


/* ------------------------------------------------------------------------ */
/* coef: gauge.F90:12-43                                                     */
/* ------------------------------------------------------------------------ */
void orc_coef(const orc_lat *L, orc_zd *u, const float *theta) {
  for (int mu = 0; mu < 3; mu++)
    for (int t = 1; t <= L->lt; t++)
      for (int y = 1; y <= L->ly; y++)
        for (int x = 1; x <= L->lx; x++) {
          /* (1.0 + cmplx(0.0, theta)) in single precision, widened (gauge.F90:27) */
          float re = 1.0f + 0.0f, im = theta[I3(x, y, t, mu)];
          u[I4(x, y, t, mu)] = zd((double)re, (double)im);
        }
  if (L->ibound == -1) { /* gauge.F90:30-32, whole slice including x/y halos */
    for (int y = 0; y <= L->ly + 1; y++)
      for (int x = 0; x <= L->lx + 1; x++) {
        orc_zd *p = &u[I4(x, y, L->lt, 2)];
        *p = zd(-p->re, -p->im);
      }
  }
  orc_update_halo_4(L, 3, u);
}

/* ------------------------------------------------------------------------ */
/* Shamir dslash / dslashd: dirac.F90:29-179, :303-407, :434-494             */
/* ------------------------------------------------------------------------ */
static void hop_shamir(const orc_lat *L, orc_zd *Phi, const orc_zd *R, const orc_zd *u, double gsign) {
  /* Wilson term (hermitian) and Dirac term (antihermitian): dirac.F90:49-76 and :464-491.
   * gsign = +1 for M, -1 for M^dagger (dirac.F90:482). Per element the mu order
   * 1,2,3 is preserved. */
#pragma omp parallel for schedule(static)
  for (int t = 1; t <= L->lt; t++)
    for (int mu = 0; mu < 3; mu++) {
      int ixup = (mu == 0), iyup = (mu == 1), itup = (mu == 2);
      for (int d = 0; d < 4; d++) {
        int g = GAM_IN[mu][d];
        orc_zd gv = gamval(mu, d);
        if (gsign < 0) gv = zd(-gv.re, -gv.im);
        for (int y = 1; y <= L->ly; y++)
          for (int x = 1; x <= L->lx; x++) {
            orc_zd uf = u[I4(x, y, t, mu)];
            orc_zd ub = zconj(u[I4(x - ixup, y - iyup, t - itup, mu)]);
            for (int s = 1; s <= L->ls; s++) {
              orc_zd rfd = R[I5(s, x + ixup, y + iyup, t + itup, d)];
              orc_zd rbd = R[I5(s, x - ixup, y - iyup, t - itup, d)];
              orc_zd rfg = R[I5(s, x + ixup, y + iyup, t + itup, g)];
              orc_zd rbg = R[I5(s, x - ixup, y - iyup, t - itup, g)];
              orc_zd w = zscal(AKAPPA, zadd(zmul(uf, rfd), zmul(ub, rbd)));
              orc_zd dd = zmul(gv, zsub(zmul(uf, rfg), zmul(ub, rbg)));
              size_t o = I5(s, x, y, t, d);
              Phi[o] = zadd(zsub(Phi[o], w), dd);
            }
          }
      }
    }
}

void orc_dslash_shamir(const orc_lat *L, orc_zd *Phi, const orc_zd *R, const orc_zd *u, float am, int imass) {
  float diag = (3.0f - L->am3) + 1.0f; /* dirac.F90:45 */
  size_t n = orc_n5(L);
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; i++) Phi[i] = zscal((double)diag, R[i]);
  hop_shamir(L, Phi, R, u, +1.0);
  /* s-like term, np_third == 1 branch: dirac.F90:80-87 */
#pragma omp parallel for schedule(static)
  for (int t = 1; t <= L->lt; t++)
    for (int y = 1; y <= L->ly; y++)
      for (int x = 1; x <= L->lx; x++) {
        for (int d = 2; d < 4; d++)
          for (int s = 1; s <= L->ls - 1; s++) Phi[I5(s, x, y, t, d)] = zsub(Phi[I5(s, x, y, t, d)], R[I5(s + 1, x, y, t, d)]);
        for (int d = 0; d < 2; d++)
          for (int s = 2; s <= L->ls; s++) Phi[I5(s, x, y, t, d)] = zsub(Phi[I5(s, x, y, t, d)], R[I5(s - 1, x, y, t, d)]);
      }
  /* mass term: dirac.F90:119-176 */
  int Ls = L->ls;
  for (int t = 1; t <= L->lt; t++)
    for (int y = 1; y <= L->ly; y++)
      for (int x = 1; x <= L->lx; x++) {
        if (imass == 1) {
          orc_zd zk = zd((double)am, 0.0);
          for (int d = 2; d < 4; d++) Phi[I5(Ls, x, y, t, d)] = zadd(Phi[I5(Ls, x, y, t, d)], zmul(zk, R[I5(Ls + 1, x, y, t, d)]));
          for (int d = 0; d < 2; d++) Phi[I5(1, x, y, t, d)] = zadd(Phi[I5(1, x, y, t, d)], zmul(zk, R[I5(0, x, y, t, d)]));
        } else if (imass == 3) {
          orc_zd zk = zd(0.0, (double)(-am));
          for (int d = 2; d < 4; d++) Phi[I5(Ls, x, y, t, d)] = zsub(Phi[I5(Ls, x, y, t, d)], zmul(zk, R[I5(Ls + 1, x, y, t, d)]));
          for (int d = 0; d < 2; d++) Phi[I5(1, x, y, t, d)] = zadd(Phi[I5(1, x, y, t, d)], zmul(zk, R[I5(0, x, y, t, d)]));
        } else if (imass == 5) {
          orc_zd zk = zd(0.0, (double)(-am));
          for (int d = 2; d < 4; d++) Phi[I5(Ls, x, y, t, d)] = zsub(Phi[I5(Ls, x, y, t, d)], zmul(zk, R[I5(Ls, x, y, t, d - 2)]));
          for (int d = 0; d < 2; d++) Phi[I5(1, x, y, t, d)] = zsub(Phi[I5(1, x, y, t, d)], zmul(zk, R[I5(1, x, y, t, d + 2)]));
        }
      }
}

void orc_dslashd_shamir(const orc_lat *L, orc_zd *Phi, const orc_zd *R, const orc_zd *u, float am, int imass) {
  /* dslashd_local_shamir: dirac.F90:303-405 */
  float diag = (3.0f - L->am3) + 1.0f;
  int Ls = L->ls;
#pragma omp parallel for schedule(static)
  for (int t = 1; t <= L->lt; t++)
    for (int d = 0; d < 4; d++)
      for (int y = 1; y <= L->ly; y++)
        for (int x = 1; x <= L->lx; x++)
          for (int s = 1; s <= Ls; s++) Phi[I5(s, x, y, t, d)] = zscal((double)diag, R[I5(s, x, y, t, d)]);
#pragma omp parallel for schedule(static)
  for (int t = 1; t <= L->lt; t++)
    for (int y = 1; y <= L->ly; y++)
      for (int x = 1; x <= L->lx; x++) {
        for (int d = 0; d < 2; d++)
          for (int s = 1; s <= Ls - 1; s++) Phi[I5(s, x, y, t, d)] = zsub(Phi[I5(s, x, y, t, d)], R[I5(s + 1, x, y, t, d)]);
        for (int d = 2; d < 4; d++)
          for (int s = 2; s <= Ls; s++) Phi[I5(s, x, y, t, d)] = zsub(Phi[I5(s, x, y, t, d)], R[I5(s - 1, x, y, t, d)]);
      }
  for (int t = 1; t <= L->lt; t++)
    for (int y = 1; y <= L->ly; y++)
      for (int x = 1; x <= L->lx; x++) {
        if (imass == 1) {
          orc_zd zk = zd((double)am, 0.0);
          for (int d = 0; d < 2; d++) Phi[I5(Ls, x, y, t, d)] = zadd(Phi[I5(Ls, x, y, t, d)], zmul(zk, R[I5(Ls + 1, x, y, t, d)]));
          for (int d = 2; d < 4; d++) Phi[I5(1, x, y, t, d)] = zadd(Phi[I5(1, x, y, t, d)], zmul(zk, R[I5(0, x, y, t, d)]));
        } else if (imass == 3) {
          orc_zd zk = zd(0.0, (double)am);
          for (int d = 0; d < 2; d++) Phi[I5(Ls, x, y, t, d)] = zadd(Phi[I5(Ls, x, y, t, d)], zmul(zk, R[I5(Ls + 1, x, y, t, d)]));
          for (int d = 2; d < 4; d++) Phi[I5(1, x, y, t, d)] = zsub(Phi[I5(1, x, y, t, d)], zmul(zk, R[I5(0, x, y, t, d)]));
        } else if (imass == 5) {
          orc_zd zk = zd(0.0, (double)am);
          for (int d = 0; d < 2; d++) Phi[I5(Ls, x, y, t, d)] = zsub(Phi[I5(Ls, x, y, t, d)], zmul(zk, R[I5(Ls, x, y, t, d + 2)]));
          for (int d = 2; d < 4; d++) Phi[I5(1, x, y, t, d)] = zsub(Phi[I5(1, x, y, t, d)], zmul(zk, R[I5(1, x, y, t, d - 2)]));
        }
      }
  hop_shamir(L, Phi, R, u, -1.0);
}

/* ------------------------------------------------------------------------ */
/* Wilson kernel: DWilson/DWilsonD on 3D slices, dirac.F90:181-301, :496-626 */
/* ------------------------------------------------------------------------ */
/* slice arrays are (0:Lx+1,0:Ly+1,0:Lt+1,4) complex(dp), i.e. I4 with c = spin */
static void dwilson(const orc_lat *L, orc_zd *Phi, const orc_zd *R, const orc_zd *u, double diag, double gsign) {
  size_t n = orc_n4(L) * 4;
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; i++) Phi[i] = zscal(diag, R[i]);
  for (int mu = 0; mu < 3; mu++) {
    int ixup = (mu == 0), iyup = (mu == 1), itup = (mu == 2);
    for (int d = 0; d < 4; d++) {
      int g = GAM_IN[mu][d];
      orc_zd gv = gamval(mu, d);
      if (gsign < 0) gv = zd(-gv.re, -gv.im);
#pragma omp parallel for schedule(static)
      for (int t = 1; t <= L->lt; t++)
        for (int y = 1; y <= L->ly; y++)
          for (int x = 1; x <= L->lx; x++) {
            orc_zd uf = u[I4(x, y, t, mu)];
            orc_zd ub = zconj(u[I4(x - ixup, y - iyup, t - itup, mu)]);
            orc_zd w = zscal(AKAPPA, zadd(zmul(uf, R[I4(x + ixup, y + iyup, t + itup, d)]),
                                          zmul(ub, R[I4(x - ixup, y - iyup, t - itup, d)])));
            orc_zd dd = zmul(gv, zsub(zmul(uf, R[I4(x + ixup, y + iyup, t + itup, g)]),
                                      zmul(ub, R[I4(x - ixup, y - iyup, t - itup, g)])));
            size_t o = I4(x, y, t, d);
            Phi[o] = zadd(zsub(Phi[o], w), dd);
          }
    }
  }
}

/* copy slice R(il,:,:,:,d0..d1) into sl (whole slice incl. halos) */
static void get_slice(const orc_lat *L, orc_zd *sl, const orc_zd *R, int il, int d0, int d1) {
  for (int d = d0; d <= d1; d++)
    for (int t = 0; t <= L->lt + 1; t++)
      for (int y = 0; y <= L->ly + 1; y++)
        for (int x = 0; x <= L->lx + 1; x++) sl[I4(x, y, t, d)] = R[I5(il, x, y, t, d)];
}

/* Phi(il, spins d0..d1, whole slice) = (Phi + a) + sg*b */
static void acc_slice(const orc_lat *L, orc_zd *Phi, int il, int d0, int d1, const orc_zd *a, const orc_zd *b,
                      double sg) {
  for (int d = d0; d <= d1; d++)
    for (int t = 0; t <= L->lt + 1; t++)
      for (int y = 0; y <= L->ly + 1; y++)
        for (int x = 0; x <= L->lx + 1; x++) {
          size_t q = I4(x, y, t, d), o = I5(il, x, y, t, d);
          orc_zd v = a ? zadd(Phi[o], a[q]) : Phi[o];
          if (b) v = (sg > 0) ? zadd(v, b[q]) : zsub(v, b[q]);
          Phi[o] = v;
        }
}

/* DWilson(Phi, R, u, mass) on one slice (dirac.F90:181-224): diag = (3.0 + mass)
 * evaluated in default real and widened; R's halos must hold the periodic images. */
void orc_dwilson(const orc_lat *L, orc_zd *Phi, const orc_zd *R, const orc_zd *u, float mass) {
  dwilson(L, Phi, R, u, (double)(3.0f + mass), +1.0);
}

void orc_dslash_wilson(const orc_lat *L, orc_zd *Phi, const orc_zd *R, const orc_zd *u, float am, int imass) {
  size_t n4 = orc_n4(L) * 4, n5 = orc_n5(L);
  int Ls = L->ls;
  double dgw = (double)(3.0f + (-L->am3)); /* DWilson diag (real(dp)) with mass = -am3: dirac.F90:191 */
  orc_zd *Rs = (orc_zd *)calloc(n4, sizeof(orc_zd));
  orc_zd *Ps = (orc_zd *)malloc(n4 * sizeof(orc_zd));
  for (size_t i = 0; i < n5; i++) Phi[i] = zd(0, 0);
  /* P+ component: dirac.F90:244-255 */
  memset(Rs, 0, n4 * sizeof(orc_zd));
  for (int il = 1; il <= Ls; il++) {
    get_slice(L, Rs, R, il, 0, 1);
    dwilson(L, Ps, Rs, u, dgw, +1.0);
    acc_slice(L, Phi, il, 0, 3, Ps, Rs, +1.0);
    if (il < Ls) acc_slice(L, Phi, il + 1, 0, 3, Ps, Rs, -1.0);
  }
  /* P- component: dirac.F90:257-268 */
  memset(Rs, 0, n4 * sizeof(orc_zd));
  for (int il = 1; il <= Ls; il++) {
    get_slice(L, Rs, R, il, 2, 3);
    dwilson(L, Ps, Rs, u, dgw, +1.0);
    acc_slice(L, Phi, il, 0, 3, Ps, Rs, +1.0);
    if (il > 1) acc_slice(L, Phi, il - 1, 0, 3, Ps, Rs, -1.0);
  }
  /* mass terms: dirac.F90:270-294 */
  for (int wall = 0; wall < 2; wall++) {
    memset(Rs, 0, n4 * sizeof(orc_zd));
    if (wall == 0) get_slice(L, Rs, R, Ls, 0, 1);
    else get_slice(L, Rs, R, 1, 2, 3);
    dwilson(L, Ps, Rs, u, dgw, +1.0);
    orc_zd c;
    if (imass == 1) c = zd((double)(-am), 0.0);
    else c = (wall == 0) ? zd(-0.0, (double)(-am)) : zd(0.0, (double)am);
    int tgt = (wall == 0) ? 1 : Ls;
    for (int d = 0; d < 4; d++)
      for (int t = 1; t <= L->lt; t++)
        for (int y = 1; y <= L->ly; y++)
          for (int x = 1; x <= L->lx; x++) {
            size_t q = I4(x, y, t, d);
            orc_zd m = zsub(Ps[q], Rs[q]);
            orc_zd ms = (imass == 1) ? zscal(c.re, m) : zmul(c, m);
            Phi[I5(tgt, x, y, t, d)] = zadd(Phi[I5(tgt, x, y, t, d)], ms);
          }
  }
  free(Rs);
  free(Ps);
}

void orc_dslashd_wilson(const orc_lat *L, orc_zd *Phi, const orc_zd *R, const orc_zd *u, float am, int imass) {
  size_t n4 = orc_n4(L) * 4, n5 = orc_n5(L);
  int Ls = L->ls;
  double dgw = (double)(float)(3.0f + (-L->am3)); /* DWilsonD diag is `real`: dirac.F90:503-505 */
  orc_zd *Rs = (orc_zd *)malloc(n4 * sizeof(orc_zd));
  orc_zd *Ps = (orc_zd *)malloc(n4 * sizeof(orc_zd));
  for (size_t i = 0; i < n5; i++) Phi[i] = zd(0, 0);
  /* dirac.F90:566-579 */
  for (int il = 1; il <= Ls; il++) {
    get_slice(L, Rs, R, il, 0, 3);
    acc_slice(L, Phi, il, 0, 3, NULL, Rs, +1.0);
    if (il < Ls) acc_slice(L, Phi, il + 1, 2, 3, NULL, Rs, -1.0);
    if (il > 1) acc_slice(L, Phi, il - 1, 0, 1, NULL, Rs, -1.0);
  }
  /* dirac.F90:582-596 */
  for (int il = 1; il <= Ls; il++) {
    get_slice(L, Rs, R, il, 0, 3);
    dwilson(L, Ps, Rs, u, dgw, -1.0);
    acc_slice(L, Phi, il, 0, 3, Ps, NULL, +1.0);
    if (il < Ls) acc_slice(L, Phi, il + 1, 2, 3, Ps, NULL, +1.0);
    if (il > 1) acc_slice(L, Phi, il - 1, 0, 1, Ps, NULL, +1.0);
  }
  /* mass terms: dirac.F90:598-622 */
  for (int wall = 0; wall < 2; wall++) {
    get_slice(L, Rs, R, wall == 0 ? Ls : 1, 0, 3);
    dwilson(L, Ps, Rs, u, dgw, -1.0);
    orc_zd zk;
    if (imass == 1) zk = zd(-(double)am, -0.0);
    else zk = (wall == 0) ? zd(-0.0, -(double)am) : zd(0.0, (double)am);
    int tgt = (wall == 0) ? 1 : Ls;
    int d0 = (wall == 0) ? 2 : 0;
    for (int d = d0; d < d0 + 2; d++)
      for (int t = 1; t <= L->lt; t++)
        for (int y = 1; y <= L->ly; y++)
          for (int x = 1; x <= L->lx; x++) {
            orc_zd m = zsub(Ps[I4(x, y, t, d)], Rs[I4(x, y, t, d)]);
            Phi[I5(tgt, x, y, t, d)] = zadd(Phi[I5(tgt, x, y, t, d)], zmul(zk, m));
          }
  }
  free(Rs);
  free(Ps);
}

void orc_dslash(const orc_lat *L, orc_zd *Phi, const orc_zd *R, const orc_zd *u, float am, int imass) {
  if (L->kernel == 1) orc_dslash_wilson(L, Phi, R, u, am, imass);
  else orc_dslash_shamir(L, Phi, R, u, am, imass);
}
void orc_dslashd(const orc_lat *L, orc_zd *Phi, const orc_zd *R, const orc_zd *u, float am, int imass) {
  if (L->kernel == 1) orc_dslashd_wilson(L, Phi, R, u, am, imass);
  else orc_dslashd_shamir(L, Phi, R, u, am, imass);
}

/* ------------------------------------------------------------------------ */
/* single-precision Shamir operators: dirac_sp.F90 as generated by           */
/* convert_to_sp.sh:14-26 from dirac.F90                                     */
/* ------------------------------------------------------------------------ */
static void hop_shamir_sp(const orc_lat *L, orc_zf *Phi, const orc_zf *R, const orc_zf *u, float gsign) {
#pragma omp parallel for schedule(static)
  for (int t = 1; t <= L->lt; t++)
    for (int mu = 0; mu < 3; mu++) {
      int ixup = (mu == 0), iyup = (mu == 1), itup = (mu == 2);
      for (int d = 0; d < 4; d++) {
        int g = GAM_IN[mu][d];
        orc_zf gv = gamvalf(mu, d);
        if (gsign < 0) gv = zf(-gv.re, -gv.im);
        for (int y = 1; y <= L->ly; y++)
          for (int x = 1; x <= L->lx; x++) {
            orc_zf uf = u[I4(x, y, t, mu)];
            orc_zf ub = fconj(u[I4(x - ixup, y - iyup, t - itup, mu)]);
            for (int s = 1; s <= L->ls; s++) {
              orc_zf w = fscal(AKAPPAF, fadd(fmulz(uf, R[I5(s, x + ixup, y + iyup, t + itup, d)]),
                                             fmulz(ub, R[I5(s, x - ixup, y - iyup, t - itup, d)])));
              orc_zf dd = fmulz(gv, fsub(fmulz(uf, R[I5(s, x + ixup, y + iyup, t + itup, g)]),
                                         fmulz(ub, R[I5(s, x - ixup, y - iyup, t - itup, g)])));
              size_t o = I5(s, x, y, t, d);
              Phi[o] = fadd(fsub(Phi[o], w), dd);
            }
          }
      }
    }
}

void orc_dslash_sp(const orc_lat *L, orc_zf *Phi, const orc_zf *R, const orc_zf *u, float am, int imass) {
  float diag = (3.0f - L->am3) + 1.0f;
  size_t n = orc_n5(L);
  int Ls = L->ls;
  for (size_t i = 0; i < n; i++) Phi[i] = fscal(diag, R[i]);
  hop_shamir_sp(L, Phi, R, u, +1.0f);
  for (int t = 1; t <= L->lt; t++)
    for (int y = 1; y <= L->ly; y++)
      for (int x = 1; x <= L->lx; x++) {
        for (int d = 2; d < 4; d++)
          for (int s = 1; s <= Ls - 1; s++) Phi[I5(s, x, y, t, d)] = fsub(Phi[I5(s, x, y, t, d)], R[I5(s + 1, x, y, t, d)]);
        for (int d = 0; d < 2; d++)
          for (int s = 2; s <= Ls; s++) Phi[I5(s, x, y, t, d)] = fsub(Phi[I5(s, x, y, t, d)], R[I5(s - 1, x, y, t, d)]);
        if (imass == 1) {
          orc_zf zk = zf(am, 0.0f);
          for (int d = 2; d < 4; d++) Phi[I5(Ls, x, y, t, d)] = fadd(Phi[I5(Ls, x, y, t, d)], fmulz(zk, R[I5(Ls + 1, x, y, t, d)]));
          for (int d = 0; d < 2; d++) Phi[I5(1, x, y, t, d)] = fadd(Phi[I5(1, x, y, t, d)], fmulz(zk, R[I5(0, x, y, t, d)]));
        } else if (imass == 3) {
          orc_zf zk = zf(0.0f, -am);
          for (int d = 2; d < 4; d++) Phi[I5(Ls, x, y, t, d)] = fsub(Phi[I5(Ls, x, y, t, d)], fmulz(zk, R[I5(Ls + 1, x, y, t, d)]));
          for (int d = 0; d < 2; d++) Phi[I5(1, x, y, t, d)] = fadd(Phi[I5(1, x, y, t, d)], fmulz(zk, R[I5(0, x, y, t, d)]));
        } else if (imass == 5) {
          orc_zf zk = zf(0.0f, -am);
          for (int d = 2; d < 4; d++) Phi[I5(Ls, x, y, t, d)] = fsub(Phi[I5(Ls, x, y, t, d)], fmulz(zk, R[I5(Ls, x, y, t, d - 2)]));
          for (int d = 0; d < 2; d++) Phi[I5(1, x, y, t, d)] = fsub(Phi[I5(1, x, y, t, d)], fmulz(zk, R[I5(1, x, y, t, d + 2)]));
        }
      }
}

void orc_dslashd_sp(const orc_lat *L, orc_zf *Phi, const orc_zf *R, const orc_zf *u, float am, int imass) {
  float diag = (3.0f - L->am3) + 1.0f;
  int Ls = L->ls;
  for (int t = 1; t <= L->lt; t++)
    for (int y = 1; y <= L->ly; y++)
      for (int x = 1; x <= L->lx; x++) {
        for (int d = 0; d < 4; d++)
          for (int s = 1; s <= Ls; s++) Phi[I5(s, x, y, t, d)] = fscal(diag, R[I5(s, x, y, t, d)]);
        for (int d = 0; d < 2; d++)
          for (int s = 1; s <= Ls - 1; s++) Phi[I5(s, x, y, t, d)] = fsub(Phi[I5(s, x, y, t, d)], R[I5(s + 1, x, y, t, d)]);
        for (int d = 2; d < 4; d++)
          for (int s = 2; s <= Ls; s++) Phi[I5(s, x, y, t, d)] = fsub(Phi[I5(s, x, y, t, d)], R[I5(s - 1, x, y, t, d)]);
        if (imass == 1) {
          orc_zf zk = zf(am, 0.0f);
          for (int d = 0; d < 2; d++) Phi[I5(Ls, x, y, t, d)] = fadd(Phi[I5(Ls, x, y, t, d)], fmulz(zk, R[I5(Ls + 1, x, y, t, d)]));
          for (int d = 2; d < 4; d++) Phi[I5(1, x, y, t, d)] = fadd(Phi[I5(1, x, y, t, d)], fmulz(zk, R[I5(0, x, y, t, d)]));
        } else if (imass == 3) {
          orc_zf zk = zf(0.0f, am);
          for (int d = 0; d < 2; d++) Phi[I5(Ls, x, y, t, d)] = fadd(Phi[I5(Ls, x, y, t, d)], fmulz(zk, R[I5(Ls + 1, x, y, t, d)]));
          for (int d = 2; d < 4; d++) Phi[I5(1, x, y, t, d)] = fsub(Phi[I5(1, x, y, t, d)], fmulz(zk, R[I5(0, x, y, t, d)]));
        } else if (imass == 5) {
          orc_zf zk = zf(0.0f, am);
          for (int d = 0; d < 2; d++) Phi[I5(Ls, x, y, t, d)] = fsub(Phi[I5(Ls, x, y, t, d)], fmulz(zk, R[I5(Ls, x, y, t, d + 2)]));
          for (int d = 2; d < 4; d++) Phi[I5(1, x, y, t, d)] = fsub(Phi[I5(1, x, y, t, d)], fmulz(zk, R[I5(1, x, y, t, d - 2)]));
        }
      }
  hop_shamir_sp(L, Phi, R, u, -1.0f);
}

/* ------------------------------------------------------------------------ */
/* inverter_utils.F90:20-54                                                  */
/* ------------------------------------------------------------------------ */
void orc_dirac_operator(const orc_lat *L, orc_zd *xout, const orc_zd *xin, const orc_zd *u, float am, int imass) {
  orc_zd *xtemp = (orc_zd *)calloc(orc_n5(L), sizeof(orc_zd));
  orc_dslash(L, xtemp, xin, u, am, imass);
  orc_update_halo_5(L, xtemp);
  orc_dslashd(L, xout, xtemp, u, am, imass);
  orc_update_halo_5(L, xout);
  free(xtemp);
}

/* ------------------------------------------------------------------------ */
/* interior reductions and updates                                           */
/* ------------------------------------------------------------------------ */
/* `body` adds into `acc`.  Each time slice is summed into its own partial and the
 * partials are added in slice order, so the result does not depend on the number
 * of threads (an OpenMP reduction clause would make it depend on the machine). */
#define FOR_INTERIOR(body)                                                            \
  do {                                                                                \
    double *part_ = (double *)calloc((size_t)L->lt, sizeof(double));                  \
    _Pragma("omp parallel for schedule(static)")                                      \
    for (int t = 1; t <= L->lt; t++) {                                                \
      double acc = 0.0;                                                               \
      for (int d = 0; d < 4; d++)                                                     \
        for (int y = 1; y <= L->ly; y++)                                              \
          for (int x = 1; x <= L->lx; x++)                                            \
            for (int s_ = 1; s_ <= L->ls; s_++) { size_t i = I5(s_, x, y, t, d); body; } \
      part_[t - 1] = acc;                                                             \
    }                                                                                 \
    for (int t = 0; t < L->lt; t++) acc += part_[t];                                  \
    free(part_);                                                                      \
  } while (0)

/* sum(abs(z)**2) over the interior, abs = hypot as Fortran's intrinsic */
static double norm2_int(const orc_lat *L, const orc_zd *a) {
  double acc = 0.0;
  FOR_INTERIOR({ double m = hypot(a[i].re, a[i].im); acc += m * m; });
  return acc;
}

/* ------------------------------------------------------------------------ */
/* congrad: measure_module.F90:9-140                                         */
/* ------------------------------------------------------------------------ */
int orc_congrad(const orc_lat *L, const orc_zd *Phi, orc_zd *X, const orc_zd *u, float res, float am, int imass,
                int niterc, int *iterations) {
  size_t n = orc_n5(L);
  orc_zd *x1 = (orc_zd *)calloc(n, sizeof(orc_zd));
  orc_zd *x2 = (orc_zd *)calloc(n, sizeof(orc_zd));
  orc_zd *p = (orc_zd *)malloc(n * sizeof(orc_zd));
  orc_zd *r = (orc_zd *)malloc(n * sizeof(orc_zd));
  /* resid = 4*ksize*ksize*ksizet*kthird*res*res as a default-real expression (:41) */
  int ivol = 4 * L->lx * L->ly * L->lt * L->ls;
  float resid = ((float)ivol * res) * res;
  int itercg = 0;
  double alphan = 0.0, betacg, betacgn, betacgd, alpha, alphad;
  memcpy(p, X, n * sizeof(orc_zd));
  memcpy(r, Phi, n * sizeof(orc_zd));
  betacgd = 1.0;
  alpha = 1.0;
  int nx;
  for (nx = 1; nx <= niterc; nx++) {
    itercg++;
    orc_dslash(L, x1, p, u, am, imass);
    if (nx != 1) {
      alphad = norm2_int(L, x1);
      alpha = alphan / alphad;
#pragma omp parallel for schedule(static)
      for (size_t i = 0; i < n; i++) X[i] = zadd(X[i], zscal(alpha, p[i]));
    }
    orc_update_halo_5(L, x1);
    orc_dslashd(L, x2, x1, u, am, imass);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) r[i] = zsub(r[i], zscal(alpha, x2[i]));
    betacgn = norm2_int(L, r);
    betacg = betacgn / betacgd;
    betacgd = betacgn;
    alphan = betacgn;
    if (nx == 1) betacg = 0.0;
    orc_update_halo_5(L, r);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) p[i] = zadd(r[i], zscal(betacg, p[i]));
    if (betacgn < (double)resid) break;
  }
  if (iterations) *iterations = nx;
  free(x1);
  free(x2);
  free(p);
  free(r);
  return itercg;
}

/* ------------------------------------------------------------------------ */
/* multishift solvers: multishift_module.F90:13-284 (DP), :289-534 (SP)      */
/* ------------------------------------------------------------------------ */
typedef struct {
  int ndiagq;
  double *zeta_i, *zeta_ii, *zeta_iii, *omegas, *gammas, *correction;
  int *flags;
  double omega, gammag, delta;
  int minishift, maxishift;
} ms_scalars;

static void ms_init(ms_scalars *c, int ndiagq, const double *anum, const double *aden) {
  c->ndiagq = ndiagq;
  c->zeta_i = (double *)malloc(ndiagq * sizeof(double));
  c->zeta_ii = (double *)malloc(ndiagq * sizeof(double));
  c->zeta_iii = (double *)calloc(ndiagq, sizeof(double));
  c->omegas = (double *)calloc(ndiagq, sizeof(double));
  c->gammas = (double *)calloc(ndiagq, sizeof(double));
  c->correction = (double *)malloc(ndiagq * sizeof(double));
  c->flags = (int *)malloc(ndiagq * sizeof(int));
  double slog = 0.0;
  for (int k = 0; k < ndiagq; k++) {
    c->correction[k] = fabs(anum[k] / aden[k]); /* :87 */
    slog += log(c->correction[k]);
  }
  double gm = exp(slog / ndiagq); /* :88 */
  for (int k = 0; k < ndiagq; k++) {
    c->correction[k] = c->correction[k] / gm;
    c->flags[k] = 1;
    c->zeta_i[k] = 1.0;
    c->zeta_ii[k] = 1.0;
    c->gammas[k] = 0.0;
  }
  c->gammag = 0.0;
  c->omega = 1.0;
  c->maxishift = ndiagq;
  c->minishift = 1;
}
static void ms_free(ms_scalars *c) {
  free(c->zeta_i); free(c->zeta_ii); free(c->zeta_iii); free(c->omegas); free(c->gammas);
  free(c->correction); free(c->flags);
}
/* after alpha: :126-135 */
static void ms_after_alpha(ms_scalars *c, double alpha, const double *aden) {
  double omega_save = c->omega;
  c->omega = -c->delta / alpha;
  for (int k = c->minishift - 1; k <= c->maxishift - 1; k++) {
    c->zeta_iii[k] = (c->zeta_i[k] * c->zeta_ii[k] * omega_save) /
                     (c->omega * c->gammag * (c->zeta_i[k] - c->zeta_ii[k]) +
                      c->zeta_i[k] * omega_save * (1.0 - aden[k] * c->omega));
    c->omegas[k] = c->omega * c->zeta_iii[k] / c->zeta_ii[k];
  }
}
/* after lambda: :143, :148-150 */
static void ms_after_lambda(ms_scalars *c, double lambda) {
  c->gammag = lambda / c->delta;
  for (int k = c->minishift - 1; k <= c->maxishift - 1; k++)
    c->gammas[k] = c->gammag * c->zeta_iii[k] * c->omegas[k] / (c->zeta_ii[k] * c->omega);
}
/* convergence and window: :230-275 */
static void ms_converge(ms_scalars *c, double lambda, float res) {
  int maxi = 0, mini = c->ndiagq + 1;
  for (int k = 1; k <= c->ndiagq; k++) {
    if (c->flags[k - 1]) {
      if (sqrt(c->delta * c->zeta_ii[k - 1] * c->zeta_ii[k - 1]) * c->correction[k - 1] < (double)res) {
        c->flags[k - 1] = 0;
      } else {
        if (k > maxi) maxi = k;
        if (k < mini) mini = k;
      }
    }
  }
  c->maxishift = maxi;
  c->minishift = mini;
  for (int k = mini - 1; k <= maxi - 1; k++) {
    c->zeta_i[k] = c->zeta_ii[k];
    c->zeta_ii[k] = c->zeta_iii[k];
  }
  c->delta = lambda;
}

static double g_last_loop_seconds = 0.0;

void orc_multishift_solver(const orc_lat *L, const orc_zd *u, float am, int imass, int ndiagq, const double *aden,
                           const double *anum, orc_zd *output, const orc_zd *input, float res, int maxcg,
                           int *cg_return, int *cg_returns) {
  size_t n = orc_n5(L), no = nout(L);
  orc_zd *r = (orc_zd *)malloc(n * sizeof(orc_zd));
  orc_zd *h = (orc_zd *)calloc(n, sizeof(orc_zd));
  orc_zd *s = (orc_zd *)calloc(n, sizeof(orc_zd));
  orc_zd *p = (orc_zd *)malloc(n * sizeof(orc_zd));
  orc_zd *sf = (orc_zd *)malloc(no * ndiagq * sizeof(orc_zd));
  memcpy(r, input, n * sizeof(orc_zd));
  memcpy(p, r, n * sizeof(orc_zd));
  ms_scalars c;
  ms_init(&c, ndiagq, anum, aden);
  c.delta = norm2_int(L, r);
  memset(output, 0, no * (size_t)L->ndiag * sizeof(orc_zd));
  for (int k = 0; k < ndiagq; k++)
    for (int d = 0; d < 4; d++)
      for (int t = 1; t <= L->lt; t++)
        for (int y = 1; y <= L->ly; y++)
          for (int x = 1; x <= L->lx; x++)
            for (int ss = 1; ss <= L->ls; ss++) sf[IO(ss, x, y, t, d, k)] = input[I5(ss, x, y, t, d)];
  int it = 0;
  const double t_loop = omp_get_wtime();
  while (c.maxishift > c.minishift - 1 && it < maxcg) {
    it++;
    orc_dslash(L, h, p, u, am, imass);
    orc_update_halo_5(L, h);
    orc_dslashd(L, s, h, u, am, imass);
    double alpha = 0.0;
    {
      double acc = 0.0;
      FOR_INTERIOR({ acc += p[i].re * s[i].re - (-p[i].im) * s[i].im; });
      alpha = acc;
    }
    ms_after_alpha(&c, alpha, aden);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) r[i] = zadd(r[i], zscal(c.omega, s[i]));
    double lambda = norm2_int(L, r);
    ms_after_lambda(&c, lambda);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) p[i] = zadd(r[i], zscal(c.gammag, p[i]));
    for (int k = c.minishift - 1; k <= c.maxishift - 1; k++) {
      double om = c.omegas[k], ga = c.gammas[k], ze = c.zeta_iii[k];
#pragma omp parallel for schedule(static)
      for (int t = 1; t <= L->lt; t++)
        for (int d = 0; d < 4; d++)
          for (int y = 1; y <= L->ly; y++)
            for (int x = 1; x <= L->lx; x++)
              for (int ss = 1; ss <= L->ls; ss++) {
                size_t o = IO(ss, x, y, t, d, k);
                output[o] = zsub(output[o], zscal(om, sf[o]));
                sf[o] = zadd(zscal(ga, sf[o]), zscal(ze, r[I5(ss, x, y, t, d)]));
              }
    }
    if (cg_returns)
      for (int k = c.minishift - 1; k <= c.maxishift - 1; k++) cg_returns[k] = it;
    ms_converge(&c, lambda, res);
    orc_update_halo_5(L, p);
  }
  *cg_return = it;
  g_last_loop_seconds = omp_get_wtime() - t_loop;
  ms_free(&c);
  free(r); free(h); free(s); free(p); free(sf);
}

/* seconds the last orc_multishift_solver spent in its iteration loop (set-up excluded) */
double orc_last_loop_seconds(void) { return g_last_loop_seconds; }

/* reduce_real_dp5d (reductions.F90:6-32): FP32 terms summed into FP64 with
 * the FIRST index outermost and the fifth innermost. */
typedef float (*term_fn)(const orc_zf *a, const orc_zf *b, size_t i);
static float term_abs2(const orc_zf *a, const orc_zf *b, size_t i) {
  (void)b;
  float m = hypotf(a[i].re, a[i].im);
  return m * m;
}
static float term_redot(const orc_zf *a, const orc_zf *b, size_t i) {
  return a[i].re * b[i].re - (-a[i].im) * b[i].im;
}
static double reduce_real_dp5d(const orc_lat *L, term_fn f, const orc_zf *a, const orc_zf *b) {
  double r = 0.0;
  for (int s = 1; s <= L->ls; s++)
    for (int x = 1; x <= L->lx; x++)
      for (int y = 1; y <= L->ly; y++)
        for (int t = 1; t <= L->lt; t++)
          for (int d = 0; d < 4; d++) r = r + (double)f(a, b, I5(s, x, y, t, d));
  return r;
}

void orc_multishift_solver_sp(const orc_lat *L, const orc_zd *udp, float am, int imass, int ndiagq, const double *aden,
                              const double *anum, orc_zd *outputdp, const orc_zd *inputdp, float res, int maxcg,
                              int *cg_return, int *cg_returns) {
  size_t n = orc_n5(L), no = nout(L), nu = orc_n4(L) * 3;
  orc_zf *u = (orc_zf *)malloc(nu * sizeof(orc_zf));
  for (size_t i = 0; i < nu; i++) u[i] = zf((float)udp[i].re, (float)udp[i].im); /* :351 */
  orc_zf *r = (orc_zf *)malloc(n * sizeof(orc_zf));
  for (size_t i = 0; i < n; i++) r[i] = zf((float)inputdp[i].re, (float)inputdp[i].im); /* :352-354 */
  orc_zf *h = (orc_zf *)calloc(n, sizeof(orc_zf));
  orc_zf *s = (orc_zf *)calloc(n, sizeof(orc_zf));
  orc_zf *p = (orc_zf *)malloc(n * sizeof(orc_zf));
  orc_zf *out = (orc_zf *)calloc(no * (size_t)L->ndiag, sizeof(orc_zf));
  orc_zf *sf = (orc_zf *)malloc(no * ndiagq * sizeof(orc_zf));
  memcpy(p, r, n * sizeof(orc_zf));
  ms_scalars c;
  ms_init(&c, ndiagq, anum, aden);
  c.delta = reduce_real_dp5d(L, term_abs2, r, NULL);
  for (int k = 0; k < ndiagq; k++)
    for (int d = 0; d < 4; d++)
      for (int t = 1; t <= L->lt; t++)
        for (int y = 1; y <= L->ly; y++)
          for (int x = 1; x <= L->lx; x++)
            for (int ss = 1; ss <= L->ls; ss++) sf[IO(ss, x, y, t, d, k)] = r[I5(ss, x, y, t, d)];
  if (cg_returns)
    for (int k = 0; k < ndiagq; k++) cg_returns[k] = 0;
  int it = 0;
  while (c.maxishift > c.minishift - 1 && it < maxcg) {
    it++;
    orc_dslash_sp(L, h, p, u, am, imass);
    orc_update_halo_5_sp(L, h);
    orc_dslashd_sp(L, s, h, u, am, imass);
    double alpha = reduce_real_dp5d(L, term_redot, p, s);
    ms_after_alpha(&c, alpha, aden);
    float omf = (float)c.omega;
    for (size_t i = 0; i < n; i++) r[i] = fadd(r[i], fscal(omf, s[i]));
    double lambda = reduce_real_dp5d(L, term_abs2, r, NULL);
    ms_after_lambda(&c, lambda);
    float gf = (float)c.gammag;
    for (size_t i = 0; i < n; i++) p[i] = fadd(r[i], fscal(gf, p[i]));
    for (int k = c.minishift - 1; k <= c.maxishift - 1; k++) {
      float om = (float)c.omegas[k], ga = (float)c.gammas[k], ze = (float)c.zeta_iii[k];
#pragma omp parallel for schedule(static)
      for (int t = 1; t <= L->lt; t++)
        for (int d = 0; d < 4; d++)
          for (int y = 1; y <= L->ly; y++)
            for (int x = 1; x <= L->lx; x++)
              for (int ss = 1; ss <= L->ls; ss++) {
                size_t o = IO(ss, x, y, t, d, k);
                out[o] = fsub(out[o], fscal(om, sf[o]));
                sf[o] = fadd(fscal(ga, sf[o]), fscal(ze, r[I5(ss, x, y, t, d)]));
              }
    }
    if (cg_returns)
      for (int k = c.minishift - 1; k <= c.maxishift - 1; k++) cg_returns[k] = it;
    ms_converge(&c, lambda, res);
    orc_update_halo_5_sp(L, p);
  }
  *cg_return = it;
  size_t ntot = no * (size_t)L->ndiag;
  for (size_t i = 0; i < ntot; i++) outputdp[i] = zd((double)out[i].re, (double)out[i].im); /* :532 */
  ms_free(&c);
  free(u); free(r); free(h); free(s); free(p); free(out); free(sf);
}

/* ------------------------------------------------------------------------ */
/* derivs: derivs_module.F90:8-410                                           */
/* ------------------------------------------------------------------------ */
static void derivs_shared(const orc_lat *L, const orc_zd *R, const orc_zd *X2, double anum, int iflag, double *dSdpi) {
  float tzi_real = 2.0f * (float)anum; /* :126 */
  size_t n3 = (size_t)L->lx * L->ly * L->lt * 3;
  double *tmp = (double *)calloc(n3, sizeof(double));
  double kap = (double)(tzi_real * (float)AKAPPA); /* tzi_real*real(akappa) in default real */
  for (int mu = 0; mu < 3; mu++) {
    int ixup = (mu == 0), iyup = (mu == 1), itup = (mu == 2);
    for (int d = 0; d < 4; d++) {
#pragma omp parallel for schedule(static)
      for (int t = 1; t <= L->lt; t++)
        for (int y = 1; y <= L->ly; y++)
          for (int x = 1; x <= L->lx; x++) {
            double sm = 0.0;
            for (int s = 1; s <= L->ls; s++) {
              orc_zd a = zmul(zconj(R[I5(s, x, y, t, d)]), X2[I5(s, x + ixup, y + iyup, t + itup, d)]);
              orc_zd b = zmul(zconj(R[I5(s, x + ixup, y + iyup, t + itup, d)]), X2[I5(s, x, y, t, d)]);
              sm += a.im - b.im;
            }
            tmp[I3(x, y, t, mu)] += kap * sm;
          }
      int g = GAM_IN[mu][d];
      orc_zd gv = gamval(mu, d);
      double sg = (iflag == 0) ? 1.0 : -1.0;
#pragma omp parallel for schedule(static)
      for (int t = 1; t <= L->lt; t++)
        for (int y = 1; y <= L->ly; y++)
          for (int x = 1; x <= L->lx; x++) {
            double sm = 0.0;
            for (int s = 1; s <= L->ls; s++) {
              orc_zd a = zmul(zconj(R[I5(s, x, y, t, d)]), X2[I5(s, x + ixup, y + iyup, t + itup, g)]);
              orc_zd b = zmul(zconj(R[I5(s, x + ixup, y + iyup, t + itup, d)]), X2[I5(s, x, y, t, g)]);
              sm += zmul(gv, zadd(a, b)).im;
            }
            if (sg > 0) tmp[I3(x, y, t, mu)] = tmp[I3(x, y, t, mu)] + (double)tzi_real * sm;
            else tmp[I3(x, y, t, mu)] = tmp[I3(x, y, t, mu)] - (double)tzi_real * sm;
          }
    }
  }
  for (size_t i = 0; i < n3; i++) dSdpi[i] = dSdpi[i] + tmp[i]; /* :194 */
  free(tmp);
}

/* derivSlice: derivs_module.F90:348-410 on masked slices
 * L-slice = R(idxL, spins lmask), R-slice = X2(idxR, spins rmask) */
static void deriv_slice(const orc_lat *L, const orc_zd *R, int idxL, int l0, int l1, const orc_zd *X2, int idxR,
                        int r0, int r1, double anum, int iflag, orc_zd cmult, double *dSdpi) {
  float tzi_real = 2.0f * (float)anum;
  double kap = (double)(tzi_real * (float)AKAPPA);
  float dmult = (iflag == 1) ? -1.0f : 1.0f;
  double tdm = (double)(tzi_real * dmult);
  const orc_zd one = zd(1.0, 0.0);
#define SL(x, y, t, d) (((d) >= l0 && (d) <= l1) ? R[I5(idxL, x, y, t, d)] : zd(0, 0))
#define SR(x, y, t, d) (((d) >= r0 && (d) <= r1) ? X2[I5(idxR, x, y, t, d)] : zd(0, 0))
  for (int mu = 0; mu < 3; mu++) {
    int ixup = (mu == 0), iyup = (mu == 1), itup = (mu == 2);
    for (int d = 0; d < 4; d++) {
      for (int t = 1; t <= L->lt; t++)
        for (int y = 1; y <= L->ly; y++)
          for (int x = 1; x <= L->lx; x++) {
            orc_zd a = zmul(zmul(zmul(cmult, zconj(SL(x, y, t, d))), one), SR(x + ixup, y + iyup, t + itup, d));
            orc_zd b = zmul(zmul(zmul(cmult, zconj(SL(x + ixup, y + iyup, t + itup, d))), one), SR(x, y, t, d));
            dSdpi[I3(x, y, t, mu)] = dSdpi[I3(x, y, t, mu)] + kap * (a.im - b.im);
          }
      int g = GAM_IN[mu][d];
      orc_zd cg = zmul(cmult, gamval(mu, d));
      for (int t = 1; t <= L->lt; t++)
        for (int y = 1; y <= L->ly; y++)
          for (int x = 1; x <= L->lx; x++) {
            orc_zd a = zmul(zmul(zconj(SL(x, y, t, d)), one), SR(x + ixup, y + iyup, t + itup, g));
            orc_zd b = zmul(zmul(zconj(SL(x + ixup, y + iyup, t + itup, d)), one), SR(x, y, t, g));
            dSdpi[I3(x, y, t, mu)] = dSdpi[I3(x, y, t, mu)] + tdm * zmul(cg, zadd(a, b)).im;
          }
    }
  }
#undef SL
#undef SR
}

void orc_derivs(const orc_lat *L, const orc_zd *R, const orc_zd *X2, double anum, int iflag, float am, int imass,
                double *dSdpi) {
  derivs_shared(L, R, X2, anum, iflag, dSdpi);
  if (L->kernel != 1) return;
  /* derivs_wilson: :41-97; derivsWilsonMass :198-249 */
  int Ls = L->ls;
  orc_zd c1 = (imass == 1) ? zd((double)(-am), 0.0) : zd(0.0, (double)(-am));
  orc_zd c2 = (imass == 1) ? zd((double)(-am), 0.0) : zd(0.0, (double)am);
  if (iflag == 1) {
    deriv_slice(L, R, 1, 0, 3, X2, Ls, 0, 1, anum, iflag, c1, dSdpi);  /* DP(1, Ls) */
    deriv_slice(L, R, Ls, 0, 3, X2, 1, 2, 3, anum, iflag, c2, dSdpi);  /* DM(Ls, 1) */
  } else if (iflag == 0) {
    deriv_slice(L, R, 1, 2, 3, X2, Ls, 0, 3, anum, iflag, c1, dSdpi);  /* MD(1, Ls) */
    deriv_slice(L, R, Ls, 0, 1, X2, 1, 0, 3, anum, iflag, c2, dSdpi);  /* PD(Ls, 1) */
  }
  orc_zd one = zd(1.0, 0.0);
  for (int il = 1; il <= Ls - 1; il++) {
    if (iflag == 1) {
      deriv_slice(L, R, il, 0, 3, X2, il + 1, 2, 3, anum, iflag, one, dSdpi);  /* DM(il, il+1) */
      deriv_slice(L, R, il + 1, 0, 3, X2, il, 0, 1, anum, iflag, one, dSdpi);  /* DP(il+1, il) */
    } else if (iflag == 0) {
      deriv_slice(L, R, il, 0, 1, X2, il + 1, 0, 3, anum, iflag, one, dSdpi);  /* PD(il, il+1) */
      deriv_slice(L, R, il + 1, 2, 3, X2, il, 0, 3, anum, iflag, one, dSdpi);  /* MD(il+1, il) */
    }
  }
}

/* ------------------------------------------------------------------------ */
/* qmrherm: qmrherm_module.F90:20-197                                        */
/* ------------------------------------------------------------------------ */
int orc_qmrherm(const orc_lat *L, const orc_zd *u, const orc_zd *Phi, orc_zd *x, float res, int *itercg, float am,
                int imass, const double *anum, const double *aden, int ndiagq, int iflag, int use_sp, int max_qmr_iters,
                int *cg_returns, double *dSdpi, orc_zd *Phi0, orc_zd *x1in) {
  if (ndiagq > L->ndiag) return -1;  /* :66-73 */
  if (L->ls % 4 != 0) return -1;     /* :75-81 */
  size_t n = orc_n5(L), no = nout(L);
  int force_dp = (L->kernel == 1);   /* :54-63 */
  orc_zd *x1 = x1in ? x1in : (orc_zd *)malloc(no * (size_t)L->ndiag * sizeof(orc_zd));
  int *cgr = (int *)calloc(ndiagq, sizeof(int));
  for (size_t i = 0; i < n; i++) x[i] = zscal(anum[0], Phi[i]); /* :83 */
  if (use_sp && !force_dp)
    orc_multishift_solver_sp(L, u, am, imass, ndiagq, aden, anum + 1, x1, Phi, res, max_qmr_iters, itercg, cgr);
  else
    orc_multishift_solver(L, u, am, imass, ndiagq, aden, anum + 1, x1, Phi, res, max_qmr_iters, itercg, cgr);
  if (cg_returns) memcpy(cg_returns, cgr, ndiagq * sizeof(int));
  if (iflag < 2) {
    for (int k = 0; k < ndiagq; k++) {
      double a = anum[k + 1];
#pragma omp parallel for schedule(static)
      for (int t = 1; t <= L->lt; t++)
        for (int d = 0; d < 4; d++)
          for (int y = 1; y <= L->ly; y++)
            for (int xx = 1; xx <= L->lx; xx++)
              for (int s = 1; s <= L->ls; s++) {
                size_t i = I5(s, xx, y, t, d);
                x[i] = zadd(x[i], zscal(a, x1[IO(s, xx, y, t, d, k)]));
              }
    }
    orc_update_halo_5(L, x);
    if (iflag == 1) {
      for (int k = 0; k < ndiagq; k++) {
        orc_zd *P = Phi0 + n * (size_t)k;
        for (int d = 0; d < 4; d++)
          for (int t = 1; t <= L->lt; t++)
            for (int y = 1; y <= L->ly; y++)
              for (int xx = 1; xx <= L->lx; xx++)
                for (int s = 1; s <= L->ls; s++) P[I5(s, xx, y, t, d)] = x1[IO(s, xx, y, t, d, k)];
        orc_update_halo_5(L, P);
      }
    }
  } else {
    orc_zd *R = (orc_zd *)calloc(n, sizeof(orc_zd));
    orc_zd *x2 = (orc_zd *)calloc(n, sizeof(orc_zd));
    for (int k = 0; k < ndiagq; k++) {
      for (int d = 0; d < 4; d++)
        for (int t = 1; t <= L->lt; t++)
          for (int y = 1; y <= L->ly; y++)
            for (int xx = 1; xx <= L->lx; xx++)
              for (int s = 1; s <= L->ls; s++) R[I5(s, xx, y, t, d)] = x1[IO(s, xx, y, t, d, k)];
      orc_update_halo_5(L, R);
      orc_dslash(L, x2, R, u, am, imass);
      orc_update_halo_5(L, x2);
      if (iflag == 2) {
        orc_derivs(L, R, x2, anum[k + 1], 0, am, imass, dSdpi);
      } else {
        double coeff = -anum[k + 1];
        memcpy(R, Phi0 + n * (size_t)k, n * sizeof(orc_zd));
        orc_derivs(L, R, x2, coeff, 0, am, imass, dSdpi);
        orc_dslash(L, x2, R, u, am, imass);
        orc_update_halo_5(L, x2);
        for (int d = 0; d < 4; d++)
          for (int t = 1; t <= L->lt; t++)
            for (int y = 1; y <= L->ly; y++)
              for (int xx = 1; xx <= L->lx; xx++)
                for (int s = 1; s <= L->ls; s++) R[I5(s, xx, y, t, d)] = x1[IO(s, xx, y, t, d, k)];
        orc_update_halo_5(L, R);
        orc_derivs(L, x2, R, coeff, 1, am, imass, dSdpi);
      }
    }
    free(R);
    free(x2);
  }
  if (!x1in) free(x1);
  free(cgr);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* random numbers: random.f90:28-126, site_random.f90:32-148                 */
/* ------------------------------------------------------------------------ */
static const uint64_t RNG_M = (2651554ULL << 24) + 15184245ULL; /* DM(2)*2^24 + DM(1) */
static const uint64_t RNG_MASK = (1ULL << 48) - 1ULL;

orc_rng *orc_rng_create(const orc_lat *L, int site) {
  orc_rng *g = (orc_rng *)calloc(1, sizeof(orc_rng));
  g->site = site;
  g->lx = L->lx; g->ly = L->ly; g->lt = L->lt;
  g->nstreams = site ? L->lx * L->ly * L->lt : 1;
  g->S = (uint64_t *)calloc(g->nstreams, sizeof(uint64_t));
  g->v = (float *)calloc((size_t)g->nstreams * 97, sizeof(float));
  g->y = (float *)calloc(g->nstreams, sizeof(float));
  g->idum = (int *)calloc(g->nstreams, sizeof(int));
  if (!site) g->S[0] = 2868876ULL * 16777216ULL + 16651885ULL; /* DATA DS (random.f90:20) */
  return g;
}
void orc_rng_destroy(orc_rng *g) {
  if (!g) return;
  free(g->S); free(g->v); free(g->y); free(g->idum); free(g);
}
static int stream_of(const orc_rng *g, int ix, int iy, int it) {
  return g->site ? (ix - 1) + g->lx * ((iy - 1) + g->ly * (it - 1)) : 0;
}
/* DRANF: exact integer arithmetic in doubles == S*M mod 2^48 */
double orc_dranf(orc_rng *g, int ix, int iy, int it) {
  int k = stream_of(g, ix, iy, it);
  g->S[k] = (g->S[k] * RNG_M) & RNG_MASK;
  return (double)g->S[k] / 281474976710656.0;
}
static float rranf(orc_rng *g, int ix, int iy, int it) { return (float)orc_dranf(g, ix, iy, it); }
/* RRANGET / G900GT: DS(2)*2^24 + DS(1), the 48-bit state as a double (site_random.f90:74-80, :114-118) */
double orc_rranget(orc_rng *g, int ix, int iy, int it) { return (double)g->S[stream_of(g, ix, iy, it)]; }
float orc_rano(orc_rng *g, int ix, int iy, int it) {
  int k = stream_of(g, ix, iy, it);
  float *v = g->v + (size_t)k * 97;
  if (g->idum[k] < 0) {
    g->idum[k] = 1;
    for (int j = 0; j < 97; j++) (void)rranf(g, ix, iy, it);
    for (int j = 0; j < 97; j++) v[j] = rranf(g, ix, iy, it);
    g->y[k] = rranf(g, ix, iy, it);
  }
  int j = 1 + (int)(97.0f * g->y[k]);
  if (j > 97) j = 97;
  if (j < 1) j = 1;
  g->y[k] = v[j - 1];
  float out = g->y[k];
  v[j - 1] = rranf(g, ix, iy, it);
  return out;
}
/* G900ST with a seed that must be an integer in [0, 2^48) */
static int set_seed(orc_rng *g, int k, double dseed) {
  if (!(dseed >= 0.0) || dseed >= 281474976710656.0 || dseed != floor(dseed)) return -1;
  g->S[k] = (uint64_t)dseed;
  return 0;
}
int orc_init_random(orc_rng *g, double seed) {
  if (!g->site) {
    if (set_seed(g, 0, seed + 0.0)) return -1; /* ip_global = 0 */
    g->idum[0] = -1;
    (void)orc_rano(g, 1, 1, 1);
    return 0;
  }
  for (int it = 1; it <= g->lt; it++)
    for (int iy = 1; iy <= g->ly; iy++)
      for (int ix = 1; ix <= g->lx; ix++) {
        /* seed_offset: site_random.f90:66-73 with ksize = Lx for both x and y */
        int off = (ix - 1) + g->lx * (iy - 1) + g->lx * g->lx * (it - 1);
        if (set_seed(g, stream_of(g, ix, iy, it), (double)off + seed)) return -1;
        g->idum[stream_of(g, ix, iy, it)] = -1;
        (void)orc_rano(g, ix, iy, it);
      }
  return 0;
}

/* Box-Muller transform.  log/sin/cos are evaluated in double precision and
 * rounded to single, so that the CUDA implementation (which calls CUDA's
 * double-precision functions) agrees bit for bit in all but a vanishing
 * fraction of draws; sqrt and the products stay in single precision as in
 * gaussian.F90:36,43-44,82,90-92. */
static const float TPI = 2.0f * 3.14159274101257324f; /* 2.0*acos(-1.0) in default real (gaussian.F90:5) */
static void gauss_common(const orc_lat *L, orc_rng *g, float *ps, float scale) {
  for (int it = 1; it <= L->lt; it++)
    for (int iy = 1; iy <= L->ly; iy++)
      for (int ix = 1; ix <= L->lx; ix++) {
        float u1 = orc_rano(g, ix, iy, it);
        float lg = (float)log((double)u1);
        ps[I4(ix, iy, it, 1)] = sqrtf(scale * lg);
      }
  for (int it = 1; it <= L->lt; it++)
    for (int iy = 1; iy <= L->ly; iy++)
      for (int ix = 1; ix <= L->lx; ix++) {
        float th = TPI * orc_rano(g, ix, iy, it);
        float sn = (float)sin((double)th), cs = (float)cos((double)th);
        float r = ps[I4(ix, iy, it, 1)];
        ps[I4(ix, iy, it, 0)] = r * sn;
        ps[I4(ix, iy, it, 1)] = r * cs;
      }
  orc_update_halo_4_real(L, 2, ps);
}
void orc_gauss0(const orc_lat *L, orc_rng *g, float *ps) { gauss_common(L, g, ps, -1.0f); }
void orc_gaussp(const orc_lat *L, orc_rng *g, float *ps) { gauss_common(L, g, ps, -2.0f); }

/* ------------------------------------------------------------------------ */
/* remez files: remez_common_subroutines.F90:6-35                            */
/* ------------------------------------------------------------------------ */
static int read_line_nums(FILE *f, double *a, double *b) {
  char buf[512];
  if (!fgets(buf, sizeof buf, f)) return -1;
  for (char *c = buf; *c; c++)
    if (*c == ',') *c = ' ';
  char *e;
  *a = strtod(buf, &e);
  if (e == buf) return -1;
  if (b) {
    char *e2;
    *b = strtod(e, &e2);
    if (e2 == e) return -1;
  }
  return 0;
}
int orc_read_remez_file(const char *path, int maxidx, double *anumA, double *anumB, double *adenA, double *adenB) {
  FILE *f = fopen(path, "r");
  if (!f) return -1;
  int rc = 0;
  for (int set = 0; set < 2 && !rc; set++) {
    double *num = set ? anumB : anumA, *den = set ? adenB : adenA;
    rc |= read_line_nums(f, &num[0], NULL);
    for (int i = 1; i <= maxidx && !rc; i++) rc |= read_line_nums(f, &num[i], &den[i - 1]);
  }
  fclose(f);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* tests/test_utils.F90:35-151 analytic fixture                              */
/* ------------------------------------------------------------------------ */
void orc_starting_state(const orc_lat *L, orc_zd *Phi, orc_zd *u, orc_zd *R, orc_zd *X, double *dSdpi_ref,
                        orc_zd *Phi0_orig) {
  const double tau = 8.0 * atan(1.0);
  int ksize = L->lx, ksizet = L->lt, kthird = L->ls;
  int idxmax = 4 * ksize * ksize * ksizet * kthird;
  float e1 = expf(1.0f);
  for (int j = 1; j <= 4; j++)
    for (int it = 1; it <= L->lt; it++)
      for (int iy = 1; iy <= L->ly; iy++)
        for (int ix = 1; ix <= L->lx; ix++)
          for (int s = 1; s <= L->ls; s++) {
            int idx = s + (ix - 1) * kthird + (iy - 1) * kthird * ksize + (it - 1) * kthird * ksize * ksize +
                      (j - 1) * kthird * ksize * ksize * ksizet;
            double b = ((double)(float)idx * tau) / (double)idxmax;
            orc_zd ex = zd(cos(b), sin(b));
            size_t i = I5(s, ix, iy, it, j - 1);
            if (Phi) Phi[i] = zscal((double)1.1f, ex);
            if (R) R[i] = zscal((double)1.3f, ex);
            if (X) X[i] = zscal((double)(0.5f * e1), ex);
            if (Phi0_orig)
              for (int l = 1; l <= 25; l++) {
                orc_zd v = zscal((double)(1.7f * e1), ex);
                Phi0_orig[i + orc_n5(L) * (size_t)(l - 1)] = zd(v.re + (double)l, v.im);
              }
          }
  for (int j = 1; j <= 3; j++)
    for (int it = 1; it <= L->lt; it++)
      for (int iy = 1; iy <= L->ly; iy++)
        for (int ix = 1; ix <= L->lx; ix++) {
          int idx = ix + (iy - 1) * ksize + (it - 1) * ksize * ksize + (j - 1) * ksize * ksize * ksizet;
          double b = ((double)(float)idx * tau) / (double)idxmax;
          if (u) u[I4(ix, iy, it, j - 1)] = zd(cos(b), sin(b));
          if (dSdpi_ref) dSdpi_ref[I3(ix, iy, it, j - 1)] = tau * cos(b);
        }
  if (u) orc_update_halo_4(L, 3, u);
  if (Phi) orc_update_halo_5(L, Phi);
  if (R) orc_update_halo_5(L, R);
  if (X) orc_update_halo_5(L, X);
  if (Phi0_orig)
    for (int l = 0; l < 25; l++) orc_update_halo_5(L, Phi0_orig + orc_n5(L) * (size_t)l);
}

/* ------------------------------------------------------------------------ */
/* RHMC: evolution.F90, force_module.F90, dwf3d_lib.F90                      */
/* ------------------------------------------------------------------------ */
static const float ONE = 1.0f;

int orc_initialise_phi(const orc_lat *L, orc_rng *g, const orc_zd *u, const orc_rational *rat, orc_zd *Phi,
                       float am, int imass, float rescga, int max_qmr_iters, orc_md_counts *cnt) {
  size_t n = orc_n5(L);
  float *ps = (float *)calloc(orc_n4(L) * 2, sizeof(float));
  orc_zd *R = (orc_zd *)calloc(n, sizeof(orc_zd));
  orc_zd *Xr = (orc_zd *)calloc(n, sizeof(orc_zd));
  for (int d = 0; d < 4; d++)
    for (int ith = 1; ith <= L->ls; ith++) {
      orc_gauss0(L, g, ps);
      for (int t = 0; t <= L->lt + 1; t++)
        for (int y = 0; y <= L->ly + 1; y++)
          for (int x = 0; x <= L->lx + 1; x++)
            R[I5(ith, x, y, t, d)] = zd((double)ps[I4(x, y, t, 0)], (double)ps[I4(x, y, t, 1)]);
    }
  orc_update_halo_5(L, R);
  int it1 = 0, it2 = 0, rc = 0;
  orc_zd *Phi0 = (orc_zd *)calloc(n * (size_t)L->ndiag, sizeof(orc_zd));
  rc |= orc_qmrherm(L, u, R, Xr, rescga, &it1, am, imass, rat->anum4, rat->aden4, rat->ndiag, 0, 0, max_qmr_iters,
                    NULL, NULL, Phi0, NULL);
  memcpy(R, Xr, n * sizeof(orc_zd));
  rc |= orc_qmrherm(L, u, R, Xr, rescga, &it2, ONE, 1, rat->bnum4, rat->bden4, rat->ndiag, 0, 0, max_qmr_iters, NULL,
                    NULL, Phi0, NULL);
  memcpy(Phi, Xr, n * sizeof(orc_zd));
  if (cnt) { cnt->ancgpf += it1; cnt->ancgpfpv += it2; }
  free(ps); free(R); free(Xr); free(Phi0);
  return rc;
}

void orc_initialise_pp(const orc_lat *L, orc_rng *g, float *pp) {
  float *ps = (float *)calloc(orc_n4(L) * 2, sizeof(float));
  for (int mu = 0; mu < 3; mu++) {
    orc_gaussp(L, g, ps);
    for (int t = 1; t <= L->lt; t++)
      for (int y = 1; y <= L->ly; y++)
        for (int x = 1; x <= L->lx; x++) pp[I3(x, y, t, mu)] = ps[I4(x, y, t, 0)];
  }
  free(ps);
}

int orc_force(const orc_lat *L, const orc_zd *u, const float *theta, const orc_rational *rat, const orc_zd *Phi,
              float res1, float am, int imass, int use_sp, int max_qmr_iters, double *dSdpi, orc_md_counts *cnt) {
  size_t n = orc_n5(L), n3 = (size_t)L->lx * L->ly * L->lt * 3;
  for (size_t i = 0; i < n3; i++) dSdpi[i] = 0.0;
  orc_zd *X2 = (orc_zd *)malloc(n * sizeof(orc_zd));
  orc_zd *Xr = (orc_zd *)calloc(n, sizeof(orc_zd));
  orc_zd *Phi0 = (orc_zd *)calloc(n * (size_t)L->ndiag, sizeof(orc_zd));
  int it = 0, rc = 0;
  memcpy(X2, Phi, n * sizeof(orc_zd));
  rc |= orc_qmrherm(L, u, X2, Xr, res1, &it, ONE, 1, rat->anum4g, rat->aden4g, rat->ndiagg, 1, use_sp, max_qmr_iters,
                    NULL, dSdpi, Phi0, NULL);
  if (cnt) cnt->ancgpv += it;
  memcpy(X2, Xr, n * sizeof(orc_zd));
  rc |= orc_qmrherm(L, u, X2, Xr, res1, &it, am, imass, rat->bnum2g, rat->bden2g, rat->ndiagg, 0, use_sp,
                    max_qmr_iters, NULL, dSdpi, Phi0, NULL);
  if (cnt) cnt->ancg += it;
  memcpy(X2, Xr, n * sizeof(orc_zd));
  rc |= orc_qmrherm(L, u, X2, Xr, res1, &it, am, imass, rat->anum2g, rat->aden2g, rat->ndiagg, 2, use_sp,
                    max_qmr_iters, NULL, dSdpi, Phi0, NULL);
  if (cnt) cnt->ancgf += it;
  rc |= orc_qmrherm(L, u, X2, Xr, res1, &it, ONE, 1, rat->anum4g, rat->aden4g, rat->ndiagg, 3, use_sp, max_qmr_iters,
                    NULL, dSdpi, Phi0, NULL);
  if (cnt) cnt->ancgfpv += it;
  if (L->ibound == -1)
    for (int y = 1; y <= L->ly; y++)
      for (int x = 1; x <= L->lx; x++) dSdpi[I3(x, y, L->lt, 2)] = -dSdpi[I3(x, y, L->lt, 2)];
  float bnf = L->beta * (float)L->nf;
  for (size_t i = 0; i < n3; i++) dSdpi[i] = dSdpi[i] + (double)(bnf * theta[i]); /* :109 */
  free(X2); free(Xr); free(Phi0);
  return rc;
}

int orc_hamilton(const orc_lat *L, const orc_zd *u, const float *theta, const float *pp, const orc_rational *rat,
                 const orc_zd *Phi, float res2, float am, int imass, int max_qmr_iters, double *h, double *hg,
                 double *hp, double *s, orc_md_counts *cnt) {
  size_t n = orc_n5(L), n3 = (size_t)L->lx * L->ly * L->lt * 3;
  if (L->strict_sums) {
    float sp = 0.0f, st = 0.0f;
    for (size_t i = 0; i < n3; i++) sp += pp[i] * pp[i];
    for (size_t i = 0; i < n3; i++) st += theta[i] * theta[i];
    *hp = (double)(0.5f * sp);
    *hg = (double)(0.5f * (float)L->nf * L->beta * st);
  } else {
    double sp = 0.0, st = 0.0;
    for (size_t i = 0; i < n3; i++) sp += (double)pp[i] * (double)pp[i];
    for (size_t i = 0; i < n3; i++) st += (double)theta[i] * (double)theta[i];
    *hp = 0.5 * sp;
    *hg = 0.5 * (double)L->nf * (double)L->beta * st;
  }
  orc_zd *R = (orc_zd *)malloc(n * sizeof(orc_zd));
  orc_zd *Xr = (orc_zd *)calloc(n, sizeof(orc_zd));
  orc_zd *Phi0 = (orc_zd *)calloc(n * (size_t)L->ndiag, sizeof(orc_zd));
  memcpy(R, Phi, n * sizeof(orc_zd));
  int it = 0, rc = 0;
  rc |= orc_qmrherm(L, u, R, Xr, res2, &it, ONE, 1, rat->anum4, rat->aden4, rat->ndiag, 0, 0, max_qmr_iters, NULL,
                    NULL, Phi0, NULL);
  if (it >= max_qmr_iters) rc |= -2; /* check_qmr_iterations: dwf3d_lib.F90:860-881 */
  if (cnt) cnt->ancghpv += it;
  memcpy(R, Xr, n * sizeof(orc_zd));
  rc |= orc_qmrherm(L, u, R, Xr, res2, &it, am, imass, rat->bnum2, rat->bden2, rat->ndiag, 0, 0, max_qmr_iters, NULL,
                    NULL, Phi0, NULL);
  if (it >= max_qmr_iters) rc |= -2;
  if (cnt) cnt->ancgh += it;
  double hf = 0.0;
  {
    double acc = 0.0;
    FOR_INTERIOR({ acc += R[i].re * Xr[i].re - (-R[i].im) * Xr[i].im; });
    hf = acc;
  }
  *h = *hg + *hp + hf;
  *s = *hg + hf;
  free(R); free(Xr); free(Phi0);
  return rc;
}

int orc_evolve_theta_pp(const orc_lat *L, orc_rng *g, orc_zd *u, float *theta, float *pp, const orc_rational *rat,
                        const orc_zd *Phi, int iterl, float dt, float res, float am, int imass, int use_sp,
                        int max_qmr_iters, int fixed_steps, int *itot, double *dSdpi, orc_md_counts *cnt) {
  size_t n3 = (size_t)L->lx * L->ly * L->lt * 3;
  int rc = orc_force(L, u, theta, rat, Phi, res, am, imass, use_sp, max_qmr_iters, dSdpi, cnt);
  float hdt = 0.5f * dt;
  for (size_t i = 0; i < n3; i++) pp[i] = pp[i] - (float)((double)hdt * dSdpi[i]); /* :142 */
  float proby = 1.0f / (float)iterl;
  int iter, nmax = fixed_steps > 0 ? fixed_steps : 4 * iterl;
  for (iter = 1; iter <= nmax; iter++) {
    for (size_t i = 0; i < n3; i++) theta[i] = theta[i] + dt * pp[i]; /* :157 */
    orc_coef(L, u, theta);
    rc |= orc_force(L, u, theta, rat, Phi, res, am, imass, use_sp, max_qmr_iters, dSdpi, cnt);
    float ytest = orc_rano(g, 1, 1, 1);
    int last = fixed_steps > 0 ? (iter == fixed_steps) : (ytest < proby);
    if (last) {
      for (size_t i = 0; i < n3; i++) pp[i] = pp[i] - (float)((double)hdt * dSdpi[i]);
      break;
    } else {
      for (size_t i = 0; i < n3; i++) pp[i] = pp[i] - (float)((double)dt * dSdpi[i]);
    }
  }
  if (itot) *itot += (iter < nmax ? iter : nmax);
  return rc;
}

int orc_trajectory(const orc_lat *L, orc_rng *g, float *theta, const orc_rational *rat, int iterl, float dt, float am,
                   int imass, float rescga, float rescgg, int use_sp, int max_qmr_iters, int fixed_steps,
                   orc_traj_result *out, orc_md_counts *cnt) {
  size_t n = orc_n5(L), n3 = (size_t)L->lx * L->ly * L->lt * 3;
  orc_zd *u = (orc_zd *)calloc(orc_n4(L) * 3, sizeof(orc_zd));
  orc_zd *Phi = (orc_zd *)calloc(n, sizeof(orc_zd));
  float *thetat = (float *)malloc(n3 * sizeof(float));
  float *pp = (float *)calloc(n3, sizeof(float));
  double *dSdpi = (double *)calloc(n3, sizeof(double));
  memcpy(thetat, theta, n3 * sizeof(float));
  orc_coef(L, u, thetat);
  int rc = orc_initialise_phi(L, g, u, rat, Phi, am, imass, rescga, max_qmr_iters, cnt);
  orc_initialise_pp(L, g, pp);
  double h0, hg, hp, s0, h1, s1;
  rc |= orc_hamilton(L, u, thetat, pp, rat, Phi, rescga, am, imass, max_qmr_iters, &h0, &hg, &hp, &s0, cnt);
  int itot = 0;
  rc |= orc_evolve_theta_pp(L, g, u, thetat, pp, rat, Phi, iterl, dt, rescgg, am, imass, use_sp, max_qmr_iters,
                            fixed_steps, &itot, dSdpi, cnt);
  rc |= orc_hamilton(L, u, thetat, pp, rat, Phi, rescga, am, imass, max_qmr_iters, &h1, &hg, &hp, &s1, cnt);
  double dH = h0 - h1;
  float y = expf((float)dH);
  int accept = 1;
  if (dH < 0.0) {
    float x = orc_rano(g, 1, 1, 1);
    if (x > y) accept = 0;
  }
  if (accept) memcpy(theta, thetat, n3 * sizeof(float));
  if (out) {
    out->h0 = h0; out->h1 = h1; out->dh = dH; out->ds = s0 - s1; out->s0 = s0; out->s1 = s1;
    out->accepted = accept; out->steps = itot; out->y = y;
  }
  free(u); free(Phi); free(thetat); free(pp); free(dSdpi);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* overlap (Zolotarev domain-wall) operator: measure_OWilson.F90             */
/* ------------------------------------------------------------------------ */
/* The coefficients coeffs(1..Ls) of prepZolo (measure_OWilson.F90:169-188):
 * setZolo + getRoots of ZOLO/zolomodule.f:26-65, :253-300 with lmin 0.1, lmax 5
 * by default.  The reference evaluates the elliptic functions by published
 * approximations, restated here so that the coefficients agree:
 *   K(k)       Hastings' polynomial approximation (Abramowitz & Stegun 17.3.34),
 *              as COMELP (ZOLO/ellipticmodule.f:114-197);
 *   sn(u|k)    descending Landen / arithmetic-geometric mean (A&S 16.4), stopped
 *              when c < 1e-7, as JELP (:19-112);
 *   arcsn(x|k) its integral by 3-point Gauss-Legendre quadrature over N panels,
 *              as arcsn (:417-438). */
static double zolo_K(double k) {
  const double m1 = 1.0 - k * k;
  if (k == 1.0) return 1.0e300;
  const double a = (((0.01451196212 * m1 + 0.03742563713) * m1 + 0.03590092383) * m1 + 0.09666344259) * m1 +
                   1.38629436112;
  const double b = (((0.00441787012 * m1 + 0.03328355346) * m1 + 0.06880248576) * m1 + 0.12498593597) * m1 + 0.5;
  return a - b * log(m1);
}
/* sn, dn of (u | modulus k) */
static void zolo_sn(double u, double k, double *sn, double *dn) {
  double r[41];
  double a0 = 1.0, b0 = sqrt(1.0 - k * k), a = 1.0;
  int n;
  for (n = 1; n <= 40; n++) {
    a = 0.5 * (a0 + b0);
    const double b = sqrt(a0 * b0), c = 0.5 * (a0 - b0);
    r[n] = c / a;
    if (c < 1.0e-7) break;
    a0 = a;
    b0 = b;
  }
  if (n > 40) n = 40;
  double ph = pow(2.0, n) * a * u, d = ph;
  for (int j = n; j >= 1; j--) {
    const double t = r[j] * sin(ph);
    d = 0.5 * (ph + atan(t / sqrt(fabs(1.0 - t * t))));
    ph = d;
  }
  *sn = sin(d);
  if (dn) *dn = sqrt(1.0 - k * k * (*sn) * (*sn));
}
static double zolo_arcsn_integrand(double x, double k) {
  return pow((1.0 + x) * (1.0 - x), -0.5) * pow((1.0 + k * x) * (1.0 - k * x), -0.5);
}
static double zolo_arcsn(double xmax, double k, int N) {
  const double dx = xmax / N, h = sqrt(3.0 / 5.0) * dx / 2.0;
  double x = dx / 2.0, acc = 0.0;
  for (int i = 0; i < N; i++) {
    const double vm = zolo_arcsn_integrand(x - h, k), v0 = zolo_arcsn_integrand(x, k),
                 vp = zolo_arcsn_integrand(x + h, k);
    acc += (5.0 / 9.0 * vm + 8.0 / 9.0 * v0 + 5.0 / 9.0 * vp) * dx / 2.0;
    x += dx;
  }
  return acc;
}
/* the product R(x) of zolomodule.f:114-123 over the N/2 factor pairs */
static double zolo_R(double x, const double *cnum, const double *cden, int nh) {
  double v = 1.0;
  for (int l = 0; l < nh; l++) v = v * (1.0 - x / cnum[l]) / (1.0 - x / cden[l]);
  return v;
}
void orc_zolo_coeffs(int N, double lmin, double lmax, double *coeffs) {
  const double beta = lmax / lmin, k = 1.0 / beta, kd = sqrt(1.0 - k) * sqrt(1.0 + k);
  const double K = zolo_K(k), Kd = zolo_K(kd);
  const int nh = N / 2;
  double *cnum = (double *)malloc((nh + 1) * sizeof(double)), *cden = (double *)malloc((nh + 1) * sizeof(double));
  for (int l = 0; l < nh; l++) { /* setInnerCoeffs, zolomodule.f:67-94 */
    double s;
    zolo_sn((2 * l + 2) * Kd / N, kd, &s, NULL);
    cnum[l] = -s / (1.0 - s) * s / (1.0 + s);
    zolo_sn((2 * l + 1) * Kd / N, kd, &s, NULL);
    cden[l] = -s / (1.0 - s) * s / (1.0 + s);
  }
  const double M = zolo_R(1.0, cnum, cden, nh); /* calcM */
  double esn, edn, dsn, ddn;                     /* calcC, :135-154 */
  zolo_sn(K, k, &esn, &edn);
  zolo_sn(Kd / N, kd, &dsn, &ddn);
  const double C = esn * ddn / (1.0 - edn * edn * dsn * dsn);
  const double lam = M / (C * zolo_R(C * C, cnum, cden, nh)); /* calcLambda */
  /* getRoots (Chiu's formula with this lambda), :196-251 */
  const double arg = sqrt((1.0 + 3.0 * lam) / ((1.0 + lam) * (1.0 + lam) * (1.0 + lam)));
  const double lk = sqrt((1.0 + lam) * (1.0 - lam));
  const double c1 = M * zolo_arcsn(arg, lk, 10000), c2 = 2.0 * Kd / N;
  for (int s = 0; s < N; s++) {
    const double v = ((s % 2) ? -c1 : c1) + ((s + 1) / 2) * c2;
    double sn;
    zolo_sn(v, kd, &sn, NULL);
    const double omega = sqrt(1.0 - kd * kd * sn * sn) / lmin;
    const double root = 1.0 / omega;
    coeffs[s] = 1.0 / root; /* coeffs = 1d0/zolo%roots (measure_OWilson.F90:182) */
  }
  free(cnum);
  free(cden);
}

/* Phi(il, spins d0..d1, interior) += c * (a[q] if a) + cb * (b[q] if b) with complex c, cb */
static void acc_slice_z(const orc_lat *L, orc_zd *Phi, int il, int d0, int d1, orc_zd c, const orc_zd *a, orc_zd cb,
                        const orc_zd *b) {
  for (int d = d0; d <= d1; d++)
    for (int t = 1; t <= L->lt; t++)
      for (int y = 1; y <= L->ly; y++)
        for (int x = 1; x <= L->lx; x++) {
          size_t q = I4(x, y, t, d), o = I5(il, x, y, t, d);
          orc_zd v = Phi[o];
          if (a) v = zadd(v, zmul(c, a[q]));
          if (b) v = zadd(v, zmul(cb, b[q]));
          Phi[o] = v;
        }
}

/* odslash, measure_OWilson.F90:14-89: DWilson(-am3) per slice with the
 * coefficients coeffs (0-based here) */
void orc_odslash(const orc_lat *L, orc_zd *Phi, const orc_zd *R, const orc_zd *u, float am, int imass,
                 const double *coeffs) {
  size_t n4 = orc_n4(L) * 4, n5 = orc_n5(L);
  int Ls = L->ls;
  double dgw = (double)(3.0f + (-L->am3));
  orc_zd *Rs = (orc_zd *)malloc(n4 * sizeof(orc_zd));
  orc_zd *Ps = (orc_zd *)malloc(n4 * sizeof(orc_zd));
  for (size_t i = 0; i < n5; i++) Phi[i] = zd(0, 0);
  const orc_zd one = zd(1.0, 0.0), mone = zd(-1.0, 0.0);
  for (int il = 1; il <= Ls; il++) { /* diagonal, :31-36 */
    get_slice(L, Rs, R, il, 0, 3);
    dwilson(L, Ps, Rs, u, dgw, +1.0);
    acc_slice_z(L, Phi, il, 0, 3, zd(coeffs[il - 1], 0.0), Ps, one, Rs);
  }
  for (int il = 1; il < Ls; il++) { /* upper diagonal, :38-47: P- R(il+1) */
    memset(Rs, 0, n4 * sizeof(orc_zd));
    get_slice(L, Rs, R, il + 1, 2, 3);
    dwilson(L, Ps, Rs, u, dgw, +1.0);
    acc_slice_z(L, Phi, il, 0, 3, zd(coeffs[il - 1], 0.0), Ps, mone, Rs);
  }
  for (int il = 2; il <= Ls; il++) { /* lower diagonal, :49-58: P+ R(il-1) */
    memset(Rs, 0, n4 * sizeof(orc_zd));
    get_slice(L, Rs, R, il - 1, 0, 1);
    dwilson(L, Ps, Rs, u, dgw, +1.0);
    acc_slice_z(L, Phi, il, 0, 3, zd(coeffs[il - 1], 0.0), Ps, mone, Rs);
  }
  /* mass terms, :60-85: -am | i am times (coeffs(1) DWilson(P+ R(Ls)) - P+ R(Ls)) into slice 1,
   * -am | -i am times (coeffs(Ls) DWilson(P- R(1)) - P- R(1)) into slice Ls */
  for (int wall = 0; wall < 2; wall++) {
    memset(Rs, 0, n4 * sizeof(orc_zd));
    if (wall == 0) get_slice(L, Rs, R, Ls, 0, 1);
    else get_slice(L, Rs, R, 1, 2, 3);
    dwilson(L, Ps, Rs, u, dgw, +1.0);
    const int tgt = wall == 0 ? 1 : Ls;
    const double cf = coeffs[tgt - 1];
    const orc_zd m = imass == 1 ? zd(-(double)am, 0.0) : (wall == 0 ? zd(0.0, (double)am) : zd(0.0, -(double)am));
    acc_slice_z(L, Phi, tgt, 0, 3, zmul(m, zd(cf, 0.0)), Ps, zmul(m, mone), Rs);
  }
  free(Rs);
  free(Ps);
}

/* odslashd, measure_OWilson.F90:91-167 */
void orc_odslashd(const orc_lat *L, orc_zd *Phi, const orc_zd *R, const orc_zd *u, float am, int imass,
                  const double *coeffs) {
  size_t n4 = orc_n4(L) * 4, n5 = orc_n5(L);
  int Ls = L->ls;
  double dgw = (double)(float)(3.0f + (-L->am3));
  orc_zd *Rs = (orc_zd *)malloc(n4 * sizeof(orc_zd));
  orc_zd *Ps = (orc_zd *)malloc(n4 * sizeof(orc_zd));
  for (size_t i = 0; i < n5; i++) Phi[i] = zd(0, 0);
  const orc_zd one = zd(1.0, 0.0), mone = zd(-1.0, 0.0);
  for (int il = 1; il <= Ls; il++) {
    get_slice(L, Rs, R, il, 0, 3);
    dwilson(L, Ps, Rs, u, dgw, -1.0);
    const orc_zd c = zd(coeffs[il - 1], 0.0);
    acc_slice_z(L, Phi, il, 0, 3, c, Ps, one, Rs);                 /* diagonal, :110-114 */
    if (il > 1) acc_slice_z(L, Phi, il - 1, 0, 1, c, Ps, mone, Rs); /* upper diagonal, :117-124 */
    if (il < Ls) acc_slice_z(L, Phi, il + 1, 2, 3, c, Ps, mone, Rs); /* lower diagonal, :127-134 */
  }
  /* mass terms, :137-160 */
  for (int wall = 0; wall < 2; wall++) {
    const int src = wall == 0 ? Ls : 1, tgt = wall == 0 ? 1 : Ls, d0 = wall == 0 ? 2 : 0;
    get_slice(L, Rs, R, src, 0, 3);
    dwilson(L, Ps, Rs, u, dgw, -1.0);
    const orc_zd zk = imass == 1 ? zd(-(double)am, 0.0) : (wall == 0 ? zd(0.0, (double)am) : zd(0.0, -(double)am));
    acc_slice_z(L, Phi, tgt, d0, d0 + 1, zmul(zk, zd(coeffs[src - 1], 0.0)), Ps, zmul(zk, mone), Rs);
  }
  free(Rs);
  free(Ps);
}

static double redot_int(const orc_lat *L, const orc_zd *a, const orc_zd *b) {
  double acc = 0.0;
  FOR_INTERIOR({ acc += a[i].re * b[i].re + a[i].im * b[i].im; });
  return acc;
}

/* congradO, measure_OWilson.F90:190-268: CG on odslash^dagger odslash starting
 * from X = Phi; returns itercg, *iterations = the loop index at exit */
int orc_congrad_o(const orc_lat *L, const orc_zd *Phi, orc_zd *X, const orc_zd *u, float res, float am, int imass,
                  const double *coeffs, int niterc, int *iterations) {
  size_t n = orc_n5(L);
  orc_zd *x1 = (orc_zd *)calloc(n, sizeof(orc_zd));
  orc_zd *x2 = (orc_zd *)calloc(n, sizeof(orc_zd));
  orc_zd *p = (orc_zd *)malloc(n * sizeof(orc_zd));
  orc_zd *r = (orc_zd *)malloc(n * sizeof(orc_zd));
  int ivol = 4 * L->lx * L->ly * L->lt * L->ls;
  float resid = ((float)ivol * res) * res; /* :214 */
  int itercg = 0, i = 0;
  memcpy(r, Phi, n * sizeof(orc_zd));
  memcpy(X, r, n * sizeof(orc_zd));
  orc_update_halo_5(L, X);
  orc_odslash(L, x1, X, u, am, imass, coeffs);
  orc_update_halo_5(L, x1);
  orc_odslashd(L, x2, x1, u, am, imass, coeffs);
#pragma omp parallel for schedule(static)
  for (size_t q = 0; q < n; q++) r[q] = zsub(Phi[q], x2[q]);
  orc_update_halo_5(L, r);
  memcpy(p, r, n * sizeof(orc_zd));
  double betacgn = norm2_int(L, r), alphan, alphad, alpha, betacg;
  if (!(betacgn < (double)resid)) {
    for (i = 1; i <= niterc; i++) {
      itercg++;
      orc_odslash(L, x1, p, u, am, imass, coeffs);
      orc_update_halo_5(L, x1);
      orc_odslashd(L, x2, x1, u, am, imass, coeffs);
      alphan = norm2_int(L, r);
      alphad = redot_int(L, p, x2);
      alpha = alphan / alphad;
#pragma omp parallel for schedule(static)
      for (size_t q = 0; q < n; q++) {
        X[q] = zadd(X[q], zscal(alpha, p[q]));
        r[q] = zsub(r[q], zscal(alpha, x2[q]));
      }
      orc_update_halo_5(L, r);
      betacgn = norm2_int(L, r);
      if (betacgn < (double)resid) break;
      betacg = betacgn / alphan;
#pragma omp parallel for schedule(static)
      for (size_t q = 0; q < n; q++) p[q] = zadd(r[q], zscal(betacg, p[q]));
      orc_update_halo_5(L, p);
    }
  }
  if (iterations) *iterations = i;
  free(x1);
  free(x2);
  free(p);
  free(r);
  return itercg;
}
