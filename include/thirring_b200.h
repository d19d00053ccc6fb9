/*
 * thirring_b200.h -- C ABI of the B200 fermion hot path for thirring-rhmc.
 *
 * A drop-in for the Fortran routines of the reference (j-ostmeyer/
 * thirring-rhmc) on the RHMC fermion path.  Every entry point keeps the
 * argument list of the Fortran routine it replaces (cited per function);
 * the module globals that routine reads or writes (trial::u, vector::X,
 * gforce::dSdpi, qmrherm_module::Phi0, random's state) become explicit
 * arguments or live in the context.  A Fortran caller binds these with
 * ISO_C_BINDING (see the shim module described alongside this header).
 *
 * Host arrays use the reference's Fortran layout and element types, halos
 * included:
 *   spinor   complex(dp) (0:Ls+1, 0:Lx+1, 0:Ly+1, 0:Lt+1, 4)        double[2*...]
 *   links    complex(dp) (0:Lx+1, 0:Ly+1, 0:Lt+1, 3)
 *   shifts   complex(dp) (Ls, Lx, Ly, Lt, 4, ndiag)   (no halo)
 *   theta,pp real        (Lx, Ly, Lt, 3)
 *   dSdpi    real(dp)    (Lx, Ly, Lt, 3)
 *   ps       real        (0:Lx+1, 0:Ly+1, 0:Lt+1, 2)
 * Input halos are ignored (neighbours are periodic, as the reference's halo
 * exchange on a 1x1x1x1 process grid makes them); output halos receive the
 * periodic images.  Scalars keep the reference's kinds: `real` -> float,
 * `real(dp)` -> double, `integer` -> int.
 *
 * Every function returns a thr_status (0 = success).  Calls on one context
 * are serialised on that context's CUDA stream and return when their
 * results are in the caller's host arrays.
 */
#ifndef THIRRING_B200_H
#define THIRRING_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference aborts the run (MPI_Abort / exit(1)) where
 * these are returned: qmrherm_module.F90:66-81, dwf3d_lib.F90:860-881. */
enum thr_status {
  THR_OK = 0,
  THR_ERR_BADARG = 1,      /* NULL pointer, bad imass, bad seed ...          */
  THR_ERR_BADSHAPE = 2,    /* Ls not a multiple of 4, ndiagq > ndiag ...     */
  THR_ERR_MAXITER = 3,     /* solver hit its iteration cap                   */
  THR_ERR_NAN = 4,         /* non-finite residual                            */
  THR_ERR_CUDA = 5,        /* CUDA runtime error                             */
  THR_ERR_NOMEM = 6,       /* device allocation failed                       */
  THR_ERR_UNSUPPORTED = 7, /* e.g. imass = 5 with the Wilson kernel          */
  THR_ERR_TIMEOUT = 8      /* a device-side wait gave up (a grid barrier of
                              the persistent multishift kernel)              */
};

enum thr_kernel { THR_SHAMIR = 0, THR_WILSON = 1 };
enum thr_layout { THR_NATURAL = 0, THR_EVEN_ODD = 1 };
enum thr_precision {
  THR_FP64 = 0,        /* everything in FP64 (the reference's DP path)                        */
  THR_FP32_REF = 1,    /* multishift_solver_sp semantics: FP32 vectors, FP64 scalars          */
  THR_MIXED_FP32 = 2,  /* FP32 inner solve, FP64 reliable residual and defect correction     */
  THR_MIXED_BF16 = 3   /* BF16 spinor storage, FP32 arithmetic, FP64 defect correction       */
};

/* Runtime replacement of params.F90:12-17 (compile-time sizes) and the
 * runtime parameters read from midout (dwf3d_lib.F90:143). */
typedef struct thr_params {
  int lx, ly, lt, ls; /* ksizex_l, ksizey_l, ksizet_l, kthird_l                         */
  int kernel;         /* thr_kernel: GENERATE_WITH_SHAMIR / _WILSON                      */
  int layout;         /* thr_layout of the device fields (results do not depend on it)   */
  int ndiag;          /* shift extent of x1/Phi0 arrays (params.F90: ndiag = 25)         */
  float am3;          /* domain-wall height                                              */
  float beta;         /* gauge coupling                                                  */
  int ibound;         /* -1: antiperiodic fermions in t                                  */
  int device;         /* CUDA device ordinal                                             */
} thr_params;

typedef struct thr_ctx thr_ctx;

/* ---- context ------------------------------------------------------------ */
int thr_create(const thr_params *p, thr_ctx **ctx);
int thr_destroy(thr_ctx *ctx);
const char *thr_status_string(int status);
/* Runtime parameter updates (params.F90:69-72 are module variables). */
int thr_set_am3(thr_ctx *ctx, float am3);
int thr_set_beta(thr_ctx *ctx, float beta);
/* Page-lock a caller array so its transfers run at full PCIe/C2C speed. */
int thr_host_register(void *ptr, unsigned long long bytes);
int thr_host_unregister(void *ptr);

/* ---- gauge.F90 ------------------------------------------------------------ */
/* coef(u, theta), gauge.F90:12-43: u = 1 + i*theta (FP32, widened), antiperiodic
 * flip of the t-links on the last time slice when ibound = -1, halo images.
 * The context keeps the result as its current links. */
int thr_coef(thr_ctx *ctx, double *u, const float *theta);
/* Make `u` (links layout) the context's current links (trial::u). */
int thr_set_links(thr_ctx *ctx, const double *u);

/* ---- dirac.F90 ------------------------------------------------------------ */
/* dslash(Phi, R, u, am, imass), dirac.F90:11-27: Phi = M R.
 * u may be NULL to use the context's current links. */
int thr_dslash(thr_ctx *ctx, double *Phi, const double *R, const double *u, float am, int imass);
/* dslashd(Phi, R, u, am, imass[, reqs_R]), dirac.F90:410-431: Phi = M^dagger R.
 * (reqs_R has no counterpart: there is no halo exchange to complete.) */
int thr_dslashd(thr_ctx *ctx, double *Phi, const double *R, const double *u, float am, int imass);

/* ---- measure_module.F90 -------------------------------------------------- */
/* congrad(Phi, res, itercg, am, imass[, iterations]), measure_module.F90:9-140:
 * CG on M^dagger M x = Phi with the context's current links.  X is the
 * module variable vector::X: initial guess in, solution out.  Stops when
 * |r|^2 < 4*Lx*Ly*Lt*Ls*res^2 or after niterc = Ls*Lx*Ly*Lt iterations
 * (then returns THR_ERR_MAXITER with X holding the last iterate, where the
 * reference writes a notice).  *iterations gets the Fortran loop index nx. */
int thr_congrad(thr_ctx *ctx, const double *Phi, double *X, float res, int *itercg, float am, int imass,
                int *iterations);

/* congrad with no allocation at all -- no counterpart in the reference.
 * For callers that cannot allocate device memory when they solve (their
 * device footprint is fixed once their fields are placed, e.g. memory owned
 * by an OpenACC/OpenMP runtime or a pool of their own, or they solve where an
 * allocation is not allowed).  Phi, X (initial guess in, solution out) and u
 * are the caller's device arrays in the device layout of this library for
 * the lattice `p` describes: spinors complex(dp) [4][Lt][Ly][Lx][Ls] (site
 * order per p->layout), links complex(dp) [3][V3].  The CG work vectors, the
 * partial sums and the scalars live in one 32 MiB array that belongs to the
 * library image (every GPU that loads the library holds it until exit), so
 * 4 * 4*Ls*Lx*Ly*Lt * 16 bytes plus a few KB must fit in 32 MiB (for
 * example 12^3 x 24 or 16^3 x 24); larger lattices return THR_ERR_BADSHAPE
 * before anything runs.  The first call on a device looks the array's device
 * address up (once per device); make that first call before any stream
 * capture.  All calls share the array: calls that overlap on the GPU (other
 * threads, other streams) race and must be serialised by the caller.
 * `stream` is a cudaStream_t (NULL = the legacy default stream); the call
 * returns when the solve has finished.  It runs no autotuning: the stencils
 * use a register budget tuned earlier in the process or the default (same
 * results either way), so nothing but the solve itself is launched on the
 * caller's stream and no CUDA event is created.  Semantics otherwise as
 * thr_congrad. */
int thr_congrad_static(const thr_params *p, const void *u, const void *Phi, void *X, float res, int *itercg,
                       float am, int imass, int *iterations, void *stream);

/* ---- batched measurement solves (no counterpart: the reference calls
 * congrad once per source, measure_module.F90:278,338,848,902,1230) ------- */
/* nrhs right-hand sides Phi(…, k) and guesses/solutions X(…, k) (consecutive
 * halo'd spinors) on the context's lattice and links, solved together: one
 * launch per operation for all of them, each with congrad's stopping rule
 * |r|^2 < 4*V*Ls*res^2 checked on its FP64 true residual.  precision:
 * THR_FP64, THR_MIXED_FP32 (FP32 correction solves, FP64 defect correction)
 * or THR_MIXED_BF16 (BF16 stencil operands, FP32 arithmetic).  itercg[k]
 * counts CG steps plus the FP64 residual passes; *outer the correction rounds. */
int thr_congrad_multi(thr_ctx *ctx, const double *Phi, double *X, int nrhs, float res, float am, int imass,
                      int precision, int *itercg, int *outer);
/* the same on FP64 device fields (nrhs consecutive fields of the device layout) */
int thr_congrad_multi_dev(thr_ctx *ctx, const void *Phi, void *X, int nrhs, float res, float am, int imass,
                          int precision, int *itercg, int *outer);
/* Independent lattices of uneven sizes (each with its own links) packed into
 * one persistent stencil launch per operation.  All share the operator kind
 * (p[i].kernel) and am3 of p[0]. */
typedef struct thr_pack thr_pack;
int thr_pack_create(int n, const thr_params *p, int device, thr_pack **pack);
int thr_pack_destroy(thr_pack *pack);
int thr_pack_upload(thr_pack *pack, int i, const double *u, const double *Phi, const double *X);
int thr_pack_congrad(thr_pack *pack, float res, float am, int imass, int precision, int *itercg, int *outer);
int thr_pack_download(thr_pack *pack, int i, double *X);
int thr_pack_zero_x(thr_pack *pack);
int thr_pack_get_stream(thr_pack *pack, void **stream);

/* measure(psibarpsi, res, aviter, am, imass[, isweep_total]),
 * measure_module.F90:142-162: the noisy estimator of psibarpsi on the current
 * links with the context's random numbers.  kernel_meas selects the
 * measurement routine the reference picks at compile time: 0 = measure_shamir
 * (:170-423, MEASURE_SHAMIR), 1 = measure_wilson (:431-670, MEASURE_WILSON;
 * imass 1 or 3), 2 = measure_wilsonKDDW (measure_OWilson.F90:646-673,
 * MEASURE_OWILSON; imass 1 or 3, THR_FP64 only): per noise four gauss0 draws,
 * each through IKDDW4 with congradO at res (the reference passes params.F90
 * respbp = 1e-6 there); parts[4n..4n+1] = Re/Im of the noise's pbp, aviter 0.  congrad runs on the context's (generation) kernel, as in the
 * reference.  knoise = params.F90 knoise (10 in the reference).  All
 * 4*knoise (Shamir) or 8*knoise (Wilson) solves run as one batched congrad
 * (precision: thr_precision; THR_FP64 is the reference's arithmetic).
 * Outputs: psibarpsi, susclsing (fort.200), aviter; optional parts[4*knoise] =
 * Re/Im psibarpsi1, Re/Im psibarpsi2 per noise (fort.100) and itercg[] per
 * solve in the reference's order. */
int thr_measure(thr_ctx *ctx, int kernel_meas, float res, float am, int imass, int knoise, int precision,
                float *psibarpsi, float *susclsing, float *aviter, double *parts, int *itercg);

/* meson(res, itercg, aviter, am, imass[, isweep_total]), measure_module.F90:684-1085
 * (SITE_RANDOM source positions, no smearing): nsource point sources on the
 * wall s = 1 (spins 3, 4), at positions drawn with rano at site (1,1,1); for
 * imass != 1 also the propagators with -am.  Outputs per time separation t =
 * 0..Lt-1 (fort.302/320/321): cpm[t], cmm[t], cpmn[2t..2t+1], cmmn[2t..2t+1]
 * (real, imaginary), chim (fort.400), itercg of the last solve, aviter.
 * nsource = 5 in the reference. */
int thr_meson(thr_ctx *ctx, float res, float am, int imass, int nsource, int precision, double *cpm, double *cmm,
              double *cpmn, double *cmmn, double *chim, int *itercg, float *aviter);

/* fermion(res, itercg, aviter, am, imass[, isweep_total]), measure_module.F90:1100-1376
 * (SITE_RANDOM source times): wall sources 1/ksize2 on a time slice at s = 1,
 * spins 3, 4.  Outputs cferm1[2t..2t+1], cferm2[2t..2t+1] (fort.500/501),
 * itercg of the last solve, aviter. */
int thr_fermion(thr_ctx *ctx, float res, float am, int imass, int nsource, int precision, double *cferm1,
                double *cferm2, int *itercg, float *aviter);

/* ---- measure_OWilson.F90: the overlap (Zolotarev domain-wall) operator ---- */
/* The coefficients coeffs(1:Ls) of prepZolo (measure_OWilson.F90:169-188,
 * ZOLO/zolomodule.f setZolo + getRoots): the Zolotarev approximation of sign(x)
 * on [lmin, lmax] with Ls roots (the reference uses lmin 0.1, lmax 5).  Host
 * only; coeffs[0..ls-1]. */
int thr_zolo_coeffs(int ls, double lmin, double lmax, double *coeffs);
/* prepZolo for this context's Ls on [lmin, lmax]; without a call the context
 * uses the reference's 0.1, 5 on first use.  thr_zolo_get copies them out. */
int thr_prep_zolo(thr_ctx *ctx, double lmin, double lmax);
int thr_zolo_get(thr_ctx *ctx, double *coeffs);
/* odslash(Phi, R, u, am, imass), measure_OWilson.F90:14-89, and
 * odslashd(Phi, R, u, am, imass[, reqs_R]), :91-167: the Wilson-kernel
 * domain-wall operator with slice il's DWilson term scaled by coeffs(il) (the
 * imass 3 walls with the module's sign).  Fortran halo'd spinors as thr_dslash;
 * u may be NULL for the current links; imass 1 or 3. */
int thr_odslash(thr_ctx *ctx, double *Phi, const double *R, const double *u, float am, int imass);
int thr_odslashd(thr_ctx *ctx, double *Phi, const double *R, const double *u, float am, int imass);
/* congradO(Phi, res, itercg, am, imass[, iterations]), measure_OWilson.F90:190-268:
 * CG on odslash^dagger odslash with the current links, starting from X = Phi
 * (X is output only, the module variable vector::x).  Stops when |r|^2 <
 * 4*Lx*Ly*Lt*Ls*res^2 or after Ls*Lx*Ly*Lt iterations (THR_ERR_MAXITER, where
 * the reference prints a warning).  *iterations gets the loop index at exit
 * (0 when the start already meets the stopping rule). */
int thr_congrad_o(thr_ctx *ctx, const double *Phi, double *X, float res, int *itercg, float am, int imass,
                  int *iterations);

/* ---- multishift_module.F90 ----------------------------------------------- */
/* multishift_solver(u, am, imass, ndiagq, aden, anum, output, input, res,
 * maxcg, cg_return[, cg_returns]), multishift_module.F90:13-284: solves
 * (M^dagger M + aden(i)) output(i) = input for i = 1..ndiagq.  output is
 * (Ls,Lx,Ly,Lt,4,ndiag) and is zeroed beyond ndiagq like the reference.
 * u may be NULL (current links).  cg_returns may be NULL. */
int thr_multishift_solver(thr_ctx *ctx, const double *u, float am, int imass, int ndiagq, const double *aden,
                          const double *anum, double *output, const double *input, float res, int maxcg,
                          int *cg_return, int *cg_returns);
/* multishift_solver_sp, multishift_module.F90:289-534: the same with FP32
 * vectors and links, FP64 scalars (its precision, not better). */
int thr_multishift_solver_sp(thr_ctx *ctx, const double *u, float am, int imass, int ndiagq, const double *aden,
                             const double *anum, double *output, const double *input, float res, int maxcg,
                             int *cg_return, int *cg_returns);

/* Multishift organisation (no counterpart in the reference, which has one):
 * 0 = every active shift field updated in every iteration, the reference's
 *     loop structure (multishift_module.F90:155-176);
 * 1 = (default) the per-shift updates of 16 iterations replayed in one pass
 *     over the shift fields from a ring of the last residuals; the same
 *     per-element arithmetic, about 8x less shift-field traffic.  The loop over
 *     batches runs on the device as one CUDA graph (a WHILE conditional node)
 *     per solve, without host round trips;
 * 2 = as 1, with the batches launched from the host one at a time (also what
 *     1 does while kernel profiling is on). */
int thr_set_solver(thr_ctx *ctx, int multishift_algo);

/* ---- qmrherm_module.F90 -------------------------------------------------- */
/* qmrherm(Phi, x, res, itercg, am, imass, anum, aden, ndiagq, iflag[, use_sp]
 * [, cg_returns]), qmrherm_module.F90:20-197, with the current links:
 *   iflag 0: x = anum(0) Phi + sum_i anum(i) (M^dagger M + aden(i))^-1 Phi
 *   iflag 1: as 0, and Phi0(…, i) = the i-th shifted solution
 *   iflag 2: x = anum(0) Phi; dSdpi += sum_i derivs(x_i, M x_i, anum(i), 0)
 *   iflag 3: x = anum(0) Phi; dSdpi += sum_i [derivs(Phi0_i, M x_i, -anum(i), 0)
 *                                            + derivs(M Phi0_i, x_i, -anum(i), 1)]
 * anum has ndiagq+1 entries (anum(0:ndiagq)).  use_sp selects the multishift
 * precision: 0 FP64; 1 the reference's single-precision multishift (FP32
 * vectors, FP64 scalars; Shamir only, as in the reference, else FP64);
 * THR_MIXED_FP32 (2) / THR_MIXED_BF16 (3) the mixed solver -- FP64 until the
 * base residual falls below a fraction of |Phi| (thr_set_mixed), then the
 * stencils, residuals and search direction in FP32 (BF16 storage with FP32
 * arithmetic) while the shifted solutions stay FP64; with the batched
 * organisation only (thr_set_solver 0 runs these modes in FP64).
 * dSdpi (gforce::dSdpi, accumulated) and Phi0 (qmrherm_module::Phi0,
 * (0:Ls+1,…,4,ndiag)) may be NULL to keep them in the context only; the
 * context always keeps the last Phi0 written by iflag 1.
 * max_qmr_iters <= 0 means the reference default 50000 (params.F90:56).
 * Returns THR_ERR_BADSHAPE where the reference aborts (:66-81). */
int thr_qmrherm(thr_ctx *ctx, const double *Phi, double *x, float res, int *itercg, float am, int imass,
                const double *anum, const double *aden, int ndiagq, int iflag, int use_sp, int *cg_returns,
                double *dSdpi, double *Phi0, int max_qmr_iters);

/* The mixed multishift's precision switch -- no counterpart in the reference.
 * The base iteration leaves FP64 for FP32 (BF16 storage) once |r| < switch *
 * |input|; defaults 1e-8 and 1e-13.  Rounding made while |r| is still large
 * stays in every shifted solution (the shifted systems have no residual of
 * their own to correct it), so a switch made too early costs accuracy, not
 * iterations; 0 never switches.  thr_mixed_switched_at returns the iteration
 * at which the last mixed solve switched (0: it finished in FP64). */
int thr_set_mixed(thr_ctx *ctx, double switch_fp32, double switch_bf16);
int thr_mixed_switched_at(thr_ctx *ctx, int *iteration);

/* ---- derivs_module.F90 --------------------------------------------------- */
/* derivs(R, X2, anum, iflag, am, imass), derivs_module.F90:8-26: adds the
 * force term of (R, X2) to dSdpi (gforce::dSdpi, (Lx,Ly,Lt,3), in/out; NULL
 * accumulates into the context's copy).  Shamir or Wilson per the context. */
int thr_derivs(thr_ctx *ctx, const double *R, const double *X2, double anum, int iflag, float am, int imass,
               double *dSdpi);

/* derivs on FP64 device fields (thr_field_create with THR_FP64) and the current
 * links, accumulating into the context's dSdpi (the one qmrherm_dev uses);
 * enqueued on the context's stream. */
int thr_derivs_dev(thr_ctx *ctx, const void *R, const void *X2, double anum, int iflag, float am, int imass);

/* ---- random.f90 / site_random.f90 / gaussian.F90 ------------------------- */
/* init_random(seed), site_random.f90:133-148 (site_streams = 1, one stream per
 * 3D site, seeded seed + x + Lx*y + Lx*Lx*t, on the device) or
 * random.f90:119-126 (site_streams = 0, one sequential stream, on the host).
 * seed must be an integer value in [0, 2^48). */
int thr_init_random(thr_ctx *ctx, double seed, int site_streams);
/* gauss0(ps), gaussian.F90:63-104: unit Gaussian pairs (variance 1/2 per
 * component); ps is (0:Lx+1,0:Ly+1,0:Lt+1,2) with periodic halos. */
int thr_gauss0(thr_ctx *ctx, float *ps);
/* gaussp(ps), gaussian.F90:14-61: variance 1 per component. */
int thr_gaussp(thr_ctx *ctx, float *ps);
/* The pseudofermion draw of initialise_phi_1flavour (evolution.F90:40-51: R(s, ., d) =
 * cmplx(gauss0) for d = 1..4, s = 1..Ls, 4 Ls gauss0 calls) into an FP64 device
 * field, site streams only; enqueued on the context's stream. */
int thr_phi_draw_dev(thr_ctx *ctx, void *R);
/* rano(yran, idum, ix, iy, it): one uniform draw from the stream of 1-based
 * site (ix,iy,it) (ignored for the global stream), random.f90:28-58. */
int thr_rano(thr_ctx *ctx, int ix, int iy, int it, float *out);

/* rranget(seed, 1, 1, 1), site_random.f90:74-80 / random.f90: the current
 * 48-bit state of site (1,1,1)'s generator (site streams) or of the global
 * generator, as the real(dp) the reference writes into checkpoints
 * (dwf3d_lib.F90:373, :474, :498). */
int thr_rranget(thr_ctx *ctx, double *seed);
/* The whole generator state (every site's 48-bit state, shuffle table, y and
 * idum, or the global stream's) as an opaque host image, so that a run can
 * resume with the identical random sequence -- no counterpart in the
 * reference, which reseeds from the checkpoint's seed on restart. */
int thr_rng_state_bytes(thr_ctx *ctx, unsigned long long *bytes);
int thr_rng_save(thr_ctx *ctx, void *host);
int thr_rng_load(thr_ctx *ctx, const void *host);

/* ---- checkpoints: dwf3d_lib.F90:618-767 (host only, no GPU) ----------- */
enum thr_con_format {
  THR_CON_SERIAL = 0,  /* unformatted sequential record: marker, theta, seed, marker (:651-653, :711-714) */
  THR_CON_MPIIO = 1    /* MPI build: theta at offset 0, seed + record length at 12V+4 (:632-649, :683-704) */
};
/* sread: theta real(Lx,Ly,Lt,3) and seed from a `con` file of either layout
 * (format returns which). */
int thr_read_con(const char *path, int lx, int ly, int lt, float *theta, double *seed, int *format);
/* swrite: write theta and seed in the given layout. */
int thr_write_con(const char *path, int lx, int ly, int lt, const float *theta, double seed, int format);
/* readseed / saveseed: the `random_seed` text file (one real(dp)). */
int thr_readseed(const char *path, double *seed);
int thr_saveseed(const char *path, double seed);

/* ---- RHMC: remez.F90, force_module.F90, evolution.F90, dwf3d_lib.F90 ----- */
/* The rational approximations read by dwf3d_lib.F90:205-209 (module remez:
 * anum2/aden2/bnum2/bden2/anum4/aden4/bnum4/bden4 with ndiag poles; module
 * remezg: the same with ndiagg poles).  anum/bnum have n+1 entries (0:n). */
int thr_set_remez(thr_ctx *ctx, int ndiag, const double *anum2, const double *aden2, const double *bnum2,
                  const double *bden2, const double *anum4, const double *aden4, const double *bnum4,
                  const double *bden4, int ndiagg, const double *anum2g, const double *aden2g,
                  const double *bnum2g, const double *bden2g, const double *anum4g, const double *aden4g,
                  const double *bnum4g, const double *bden4g);
/* Inverter residuals rescga (Hamiltonian, pseudofermion), rescgg (guidance)
 * and spmd (single-precision guidance solves), params.F90:60-64; defaults
 * 1e-8, 1e-6, 1.  spmd is qmrherm's use_sp for the guidance (force) solves:
 * 0 FP64, 1 the reference's single-precision multishift, THR_MIXED_FP32 /
 * THR_MIXED_BF16 the mixed multishift.  max_qmr_iters <= 0 keeps 50000. */
int thr_set_residuals(thr_ctx *ctx, float rescga, float rescgg, int spmd, int max_qmr_iters);
/* Precision of the Hamiltonian and pseudofermion solves (dwf3d_lib.F90:584,590,
 * evolution.F90:64,69), which the reference always runs in FP64: THR_FP64
 * (default), THR_MIXED_FP32 or THR_MIXED_BF16 (the mixed multishift, whose
 * precision switch keeps its rounding below FP64's; thr_set_mixed) -- no
 * counterpart in the reference. */
int thr_set_action_precision(thr_ctx *ctx, int precision);
/* force(Phi, res1, am, imass), force_module.F90:9-113, with the current
 * links; theta (trial::theta) feeds the gauge term; dSdpi is overwritten. */
int thr_force(thr_ctx *ctx, const double *Phi, float res1, float am, int imass, const float *theta, double *dSdpi);
/* hamilton(Phi, h, hg, hp, s, res2, am, imass), dwf3d_lib.F90:511-616, with
 * the current links, theta and pp (trial::theta, trial::pp).  hp and hg are
 * accumulated in FP64 (the reference sums them in single precision). */
int thr_hamilton(thr_ctx *ctx, const double *Phi, double *h, double *hg, double *hp, double *s, float res2,
                 float am, int imass, const float *theta, const float *pp);
/* initialise_phi_1flavour(phi, am, imass), evolution.F90:7-75 (site streams). */
int thr_initialise_phi(thr_ctx *ctx, double *Phi, float am, int imass);
/* initialise_pp(pp), evolution.F90:77-111 (site streams). */
int thr_initialise_pp(thr_ctx *ctx, float *pp);
/* evolve_theta_pp(iterl, dt, pp, phi, res, am, imass, itot), evolution.F90:113-179.
 * theta (trial::theta) and pp in/out; u (trial::u) and dSdpi receive the final
 * links and force when non-NULL.  fixed_steps > 0 replaces the random length by
 * exactly that many steps (the exit draw at site (1,1,1) is still consumed). */
int thr_evolve_theta_pp(thr_ctx *ctx, int iterl, float dt, float *pp, const double *Phi, float res, float am,
                        int imass, int *itot, float *theta, double *u, double *dSdpi, int fixed_steps);
/* One trajectory of the sweep loop, dwf3d_lib.F90:265-323: coef, pseudofermion
 * and momentum refresh, H0, leapfrog, H1, Metropolis.  theta is replaced by
 * the new field when accepted. */
typedef struct thr_traj_result {
  double h0, h1, dh, ds, s0, s1;
  int accepted, steps;
  float y;
} thr_traj_result;
int thr_trajectory(thr_ctx *ctx, float *theta, int iterl, float dt, float am, int imass, int fixed_steps,
                   thr_traj_result *out);
/* Solver iteration sums (counters.F90): ancg, ancgpv, ancgf, ancgfpv, ancgh,
 * ancghpv, ancgpf, ancgpfpv. */
int thr_md_counters(thr_ctx *ctx, double *counts8, int reset);

/* ---- device-resident fields ------------------------------------------- */
/* Spinor fields kept in HBM in the device layout (no halos), so that solver
 * and MD loops never cross PCIe.  `precision` is a thr_precision storage
 * choice: THR_FP64 (complex double), THR_FP32_REF (complex float) or
 * THR_MIXED_BF16 (bf16 pairs).  Operations on device fields are enqueued on
 * the context's CUDA stream and return without synchronising; thr_sync()
 * waits for them.  No counterpart in the reference (its fields are module
 * arrays in host memory). */
int thr_field_create(thr_ctx *ctx, int precision, void **field);
int thr_field_destroy(thr_ctx *ctx, void *field);
int thr_field_upload(thr_ctx *ctx, void *field, int precision, const double *host_spinor);
int thr_field_download(thr_ctx *ctx, double *host_spinor, const void *field, int precision);
/* out = M in (dag = 0) or M^dagger in (dag = 1) with the current links */
int thr_dslash_dev(thr_ctx *ctx, void *out, const void *in, int precision, float am, int imass, int dag);
/* out = odslash in (dag = 0) or odslashd in (dag = 1), FP64 fields, current links */
int thr_odslash_dev(thr_ctx *ctx, void *out, const void *in, float am, int imass, int dag);
/* qmrherm on FP64 device fields (the device layout of thr_field_create with
 * THR_FP64): same semantics as thr_qmrherm; dSdpi and Phi0 stay in the
 * context.  Returns when the solve has converged (its scalars are polled). */
int thr_qmrherm_dev(thr_ctx *ctx, const void *Phi, void *x, float res, int *itercg, float am, int imass,
                    const double *anum, const double *aden, int ndiagq, int iflag, int use_sp, int *cg_returns);
/* The solvers' fused stencil epilogues on device fields of one precision, so a
 * caller can build its own iteration from them -- no counterpart in the
 * reference.  With Op = M (dag = 0) or M^dagger (dag = 1) and the current links:
 *   mode 0: out = Op in                  (*norm2 = |out|^2 when norm2 != NULL)
 *   mode 1: out = aux + coef * Op in     (*norm2 = |out|^2; Op in is never stored)
 *   mode 3: out = Op in + coef * aux     (*norm2 = |out|^2)
 * aux must differ from in and out.  |out|^2 is summed in FP64 in a fixed order.
 * Returns after the sum is on the host (mode 0 without norm2: enqueued only). */
int thr_dslash_fused_dev(thr_ctx *ctx, void *out, const void *in, const void *aux, double coef, int precision,
                         float am, int imass, int dag, int mode, double *norm2);
/* The true residual of every shifted system, r2[k] = |Phi - (M^dagger M + aden[k]) x_k|^2
 * in FP64 for k < nq, with the current links -- no counterpart in the reference,
 * whose stopping rule (multishift_module.F90:244) tests the recursive residual.
 * Phi and x are FP64 device fields (x: nq consecutive fields); x = NULL takes the
 * context's last multishift solutions (those of the last qmrherm call). */
int thr_shift_residuals_dev(thr_ctx *ctx, const void *Phi, const void *x, int nq, const double *aden, float am,
                            int imass, double *r2);
int thr_sync(thr_ctx *ctx);
/* the context's cudaStream_t, for event timing by the caller */
int thr_get_stream(thr_ctx *ctx, void **stream);
/* Kernel timing inside the multishift solvers.  thr_profile(ctx, stride, reset):
 * stride 0 turns it off; stride k >= 1 brackets every k-th launch of each kind
 * with CUDA events on the context's stream -- kind 0 the stencil M (in the
 * batched multishift with its fused |M p|^2), kind 2 the stencil M^dagger
 * (kind 0 in the per-iteration multishift), kind 1 the shift-field update
 * (k_flush, or k_ms_pshift in the per-iteration solver), kinds 3 and 4 the
 * stencils M and M^dagger of the mixed multishift's low-precision phase, kinds 5
 * and 6 the batched multishift's one-block scalar steps k_alpha and k_lambda (no
 * algorithmic bytes).  thr_profile_read
 * returns, for one kind, the sampled launches that did work, their summed
 * device time in ms and their summed algorithmic bytes, and the number of
 * launches of that kind that did work (sampled or not). */
int thr_profile(thr_ctx *ctx, int stride, int reset);
int thr_profile_read(thr_ctx *ctx, int kind, int *sampled, double *ms, double *bytes, double *launches);

/* Blocks of the staged-tile FP64 stencil (THR_TILE=1) whose tile copies did not
 * arrive within the kernel's bounded wait (0.2 s), since the library was loaded,
 * on the context's device.  Such a block writes NaN to all its outputs and to its
 * epilogue sum, so solvers stop with THR_ERR_NAN.  No counterpart in the reference. */
int thr_stencil_timeouts(thr_ctx *ctx, unsigned long long *count);
/* The stencil autotuner's choices so far (process-wide), as text: one line per
 * tuned case with the candidates' mean launch times.  The tuner picks the
 * register budget (resident blocks per SM) of the Shamir and Wilson stencils
 * per lattice on first use (results are identical for every choice);
 * THR_TUNE=0 in the environment disables it. */
int thr_tune_report(char *buf, int len);

#ifdef __cplusplus
}
#endif
#endif
