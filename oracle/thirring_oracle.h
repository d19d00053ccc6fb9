/*
 * thirring_oracle.h -- CPU restatement of the thirring-rhmc fermion hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the CUDA
 * implementation and the timed CPU baseline.  Only the test suite, the smoke
 * check and the CPU-baseline leg of the benchmark may load it; the product
 * library never links or calls it.
 *
 * Every routine restates one Fortran routine of the reference (j-ostmeyer/
 * thirring-rhmc) on arrays in the reference's own Fortran layout, halos
 * included:
 *   spinor  (0:Ls+1, 0:Lx+1, 0:Ly+1, 0:Lt+1, 4)   complex(dp)      dirac.F90:13-15
 *   links   (0:Lx+1, 0:Ly+1, 0:Lt+1, 3)           complex(dp)      trial.F90:6
 *   theta, pp (Lx, Ly, Lt, 3)                     real             trial.F90:7-8
 *   dSdpi   (Lx, Ly, Lt, 3)                       real(dp)         gforce.F90:6
 *   ps      (0:Lx+1, 0:Ly+1, 0:Lt+1, 2)           real             dum1.F90:6
 *   shift outputs (Ls, Lx, Ly, Lt, 4, ndiag)      complex(dp)      multishift_module.F90:29
 * Complex numbers are (re, im) pairs of double / float, as in Fortran.
 *
 * Semantics are those of the MPI build on a 1x1x1x1 process grid: every halo
 * exchange is a periodic copy of the opposite face, the fifth dimension
 * included (comms.F90:67-68, comms5.F90:135-194).
 *
 * Parity is pinned against the reference's own known-answer tests
 * (tests/test_gauss0.F90:140-142, tests/test_gaussp.F90:84-86,
 * tests/test_congrad.F90:47) and the con_12x12x12 fixture; the reference's
 * snapshot .dat files are not shipped with it.
 */
#ifndef THIRRING_ORACLE_H
#define THIRRING_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double re, im; } orc_zd;
typedef struct { float re, im; } orc_zf;

/* Runtime stand-in for the compile-time and runtime parameters of
 * params.F90:12-17 (sizes), :60-62 (residuals) and the midout values. */
typedef struct orc_lat {
  int lx, ly, lt, ls;   /* ksizex_l, ksizey_l, ksizet_l, kthird_l          */
  int kernel;           /* 0 = Shamir (GENERATE_WITH_SHAMIR), 1 = Wilson    */
  int ndiag;            /* leading extent of Phi0 / x1 (params.F90:18)      */
  float am3;            /* domain-wall height (params.F90:71)               */
  float beta;           /* gauge coupling (params.F90:70)                   */
  int ibound;           /* -1 = antiperiodic in t (params.F90:72)           */
  int nf;               /* Nf (params.F90:19), 1                             */
  int strict_sums;      /* 1 = FP32 Hamiltonian sums as in dwf3d_lib.F90:542,551 */
} orc_lat;

/* sizes */
size_t orc_n5(const orc_lat *L);   /* elements of one halo'd spinor */
size_t orc_n4(const orc_lat *L);   /* elements of one halo'd 3D field component */

/* gammamatrices.F90:17-132, values already multiplied by akappa */
void orc_gammas(int mu, int d, orc_zd *val, int *gin);

/* halo updates: periodic face copies (uncomms5.f90:6-20 generalised to the
 * fifth dimension as the MPI build does) */
void orc_update_halo_5(const orc_lat *L, orc_zd *a);
void orc_update_halo_5_sp(const orc_lat *L, orc_zf *a);
void orc_update_halo_4(const orc_lat *L, int n, orc_zd *u);
/* DWilson on one (0:Lx+1,0:Ly+1,0:Lt+1,4) slice, dirac.F90:181-224 */
void orc_dwilson(const orc_lat *L, orc_zd *Phi, const orc_zd *R, const orc_zd *u, float mass);
void orc_update_halo_4_real(const orc_lat *L, int n, float *ps);

/* gauge.F90:12-43 */
void orc_coef(const orc_lat *L, orc_zd *u, const float *theta);

/* dirac.F90 */
void orc_dslash(const orc_lat *L, orc_zd *Phi, const orc_zd *R, const orc_zd *u, float am, int imass);
void orc_dslashd(const orc_lat *L, orc_zd *Phi, const orc_zd *R, const orc_zd *u, float am, int imass);
void orc_dslash_sp(const orc_lat *L, orc_zf *Phi, const orc_zf *R, const orc_zf *u, float am, int imass);
void orc_dslashd_sp(const orc_lat *L, orc_zf *Phi, const orc_zf *R, const orc_zf *u, float am, int imass);

/* inverter_utils.F90:20-54  xout = M^dagger M xin (halos refreshed) */
void orc_dirac_operator(const orc_lat *L, orc_zd *xout, const orc_zd *xin, const orc_zd *u, float am, int imass);

/* measure_module.F90:9-140; X is in/out (initial guess and solution).
 * Returns itercg; *iterations gets nx (which exceeds niterc on failure). */
int orc_congrad(const orc_lat *L, const orc_zd *Phi, orc_zd *X, const orc_zd *u,
                float res, float am, int imass, int niterc, int *iterations);

/* multishift_module.F90:13-284 and :289-534.  output is (Ls,Lx,Ly,Lt,4,ndiag). */
void orc_multishift_solver(const orc_lat *L, const orc_zd *u, float am, int imass, int ndiagq,
                           const double *aden, const double *anum, orc_zd *output,
                           const orc_zd *input, float res, int maxcg, int *cg_return,
                           int *cg_returns);
void orc_multishift_solver_sp(const orc_lat *L, const orc_zd *u, float am, int imass, int ndiagq,
                              const double *aden, const double *anum, orc_zd *output,
                              const orc_zd *input, float res, int maxcg, int *cg_return,
                              int *cg_returns);

/* derivs_module.F90:8-410; accumulates into dSdpi */
void orc_derivs(const orc_lat *L, const orc_zd *R, const orc_zd *X2, double anum, int iflag,
                float am, int imass, double *dSdpi);

/* qmrherm_module.F90:20-197.  anum has ndiagq+1 entries (anum(0:ndiagq)).
 * Phi0 is (0:Ls+1,...,4,ndiag) and persists across calls; x1 scratch
 * (Ls,Lx,Ly,Lt,4,ndiag) may be NULL.  Returns 0, or -1 on the reference's
 * abort conditions (qmrherm_module.F90:66-81). */
int orc_qmrherm(const orc_lat *L, const orc_zd *u, const orc_zd *Phi, orc_zd *x, float res,
                int *itercg, float am, int imass, const double *anum, const double *aden,
                int ndiagq, int iflag, int use_sp, int max_qmr_iters, int *cg_returns,
                double *dSdpi, orc_zd *Phi0, orc_zd *x1);

/* Random numbers.  site_random.f90 (one stream per 3D site) or random.f90
 * (one global stream).  State layout per stream: S (48-bit), v[97], y, idum. */
typedef struct orc_rng {
  int site;          /* 1 = site_random.f90, 0 = random.f90 */
  int lx, ly, lt;
  int nstreams;
  uint64_t *S;       /* DS(2) packed: S = DS(2)*2^24 + DS(1) */
  float *v;          /* 97 per stream */
  float *y;          /* yran */
  int *idum;
} orc_rng;
orc_rng *orc_rng_create(const orc_lat *L, int site);
void orc_rng_destroy(orc_rng *g);
int orc_init_random(orc_rng *g, double seed);                 /* random.f90:119 / site_random.f90:133 */
float orc_rano(orc_rng *g, int ix, int iy, int it);          /* 1-based site; ignored for global */
double orc_dranf(orc_rng *g, int ix, int iy, int it);
double orc_rranget(orc_rng *g, int ix, int iy, int it);
void orc_gauss0(const orc_lat *L, orc_rng *g, float *ps);     /* gaussian.F90:63-104 */
void orc_gaussp(const orc_lat *L, orc_rng *g, float *ps);     /* gaussian.F90:14-61 */

/* remez_common_subroutines.F90:20-35 */
int orc_read_remez_file(const char *path, int maxidx, double *anumA, double *anumB,
                        double *adenA, double *adenB);

/* tests/test_utils.F90:35-151 analytic starting state (any pointer may be NULL) */
void orc_starting_state(const orc_lat *L, orc_zd *Phi, orc_zd *u, orc_zd *R, orc_zd *X,
                        double *dSdpi_ref, orc_zd *Phi0_orig);

/* RHMC pieces (Shamir or Wilson per L->kernel) */
typedef struct orc_rational {
  int ndiag, ndiagg;
  double *anum2, *aden2, *bnum2, *bden2, *anum4, *aden4, *bnum4, *bden4;        /* 0:ndiag */
  double *anum2g, *aden2g, *bnum2g, *bden2g, *anum4g, *aden4g, *bnum4g, *bden4g; /* 0:ndiagg */
} orc_rational;

typedef struct orc_md_counts { double ancg, ancgpv, ancgf, ancgfpv, ancgh, ancghpv, ancgpf, ancgpfpv; } orc_md_counts;

/* evolution.F90:7-75 */
int orc_initialise_phi(const orc_lat *L, orc_rng *g, const orc_zd *u, const orc_rational *rat,
                       orc_zd *Phi, float am, int imass, float rescga, int max_qmr_iters, orc_md_counts *cnt);
/* evolution.F90:77-111 */
void orc_initialise_pp(const orc_lat *L, orc_rng *g, float *pp);
/* force_module.F90:9-113 */
int orc_force(const orc_lat *L, const orc_zd *u, const float *theta, const orc_rational *rat,
              const orc_zd *Phi, float res1, float am, int imass, int use_sp, int max_qmr_iters,
              double *dSdpi, orc_md_counts *cnt);
/* dwf3d_lib.F90:511-616 */
int orc_hamilton(const orc_lat *L, const orc_zd *u, const float *theta, const float *pp,
                 const orc_rational *rat, const orc_zd *Phi, float res2, float am, int imass,
                 int max_qmr_iters, double *h, double *hg, double *hp, double *s, orc_md_counts *cnt);
/* evolution.F90:113-179.  fixed_steps > 0 replaces the random trajectory
 * length by exactly that many steps (the exit draw is still consumed). */
int orc_evolve_theta_pp(const orc_lat *L, orc_rng *g, orc_zd *u, float *theta, float *pp,
                        const orc_rational *rat, const orc_zd *Phi, int iterl, float dt,
                        float res, float am, int imass, int use_sp, int max_qmr_iters,
                        int fixed_steps, int *itot, double *dSdpi, orc_md_counts *cnt);
/* one trajectory of dwf3d_lib.F90:251-323 (coef .. Metropolis) */
typedef struct orc_traj_result { double h0, h1, dh, ds, s0, s1; int accepted; int steps; float y; } orc_traj_result;
int orc_trajectory(const orc_lat *L, orc_rng *g, float *theta, const orc_rational *rat,
                   int iterl, float dt, float am, int imass, float rescga, float rescgg, int use_sp,
                   int max_qmr_iters, int fixed_steps, orc_traj_result *out, orc_md_counts *cnt);

/* overlap operator, measure_OWilson.F90: the Zolotarev coefficients of prepZolo
 * (:169-188, ZOLO/zolomodule.f) for N = Ls slices on [lmin, lmax]; odslash (:14-89),
 * odslashd (:91-167) and congradO (:190-268) with coefficients coeffs[0..Ls-1] */
void orc_zolo_coeffs(int N, double lmin, double lmax, double *coeffs);
void orc_odslash(const orc_lat *L, orc_zd *Phi, const orc_zd *R, const orc_zd *u, float am, int imass,
                 const double *coeffs);
void orc_odslashd(const orc_lat *L, orc_zd *Phi, const orc_zd *R, const orc_zd *u, float am, int imass,
                  const double *coeffs);
int orc_congrad_o(const orc_lat *L, const orc_zd *Phi, orc_zd *X, const orc_zd *u, float res, float am, int imass,
                  const double *coeffs, int niterc, int *iterations);

/* threads used by the OpenMP loops */
int orc_num_threads(void);
/* seconds the last orc_multishift_solver spent in its iteration loop (set-up excluded) */
double orc_last_loop_seconds(void);
void orc_set_num_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
