// ctx.h -- the device context behind a thr_ctx handle.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "../../include/thirring_b200.h"
#include "rng.h"
#include "thr_common.cuh"
#include "thr_kernels.h"

#define THR_CUDA(call)                                 \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return THR_ERR_CUDA;   \
  } while (0)
#define THR_TRY(...)                  \
  do {                                \
    int rc_ = (__VA_ARGS__);          \
    if (rc_ != THR_OK) return rc_;    \
  } while (0)

// slots of the context's device scalar block (dscal, 4096 doubles) outside the
// solver states that start at its base
constexpr int kScalHamSum = 4000;      // hamilton's fermion sum
constexpr int kScalFusedCoef = 4090;   // thr_dslash_fused_dev: the epilogue coefficient
constexpr int kScalFusedSum = 4091;    // thr_dslash_fused_dev / thr_shift_residuals_dev: a reduced sum
constexpr int kScalMd = 4064;          // MD step graph: 8 iteration counters, then its control block
constexpr int kMsTemplates = 8;        // multishift state templates of one captured MD step
constexpr int kIscalChainBar = 0;      // iscal[0..2]: the persistent multishift kernel's barrier words

struct thr_ctx {
  thr_params p;
  thr::Geom g;
  int dev = 0;
  cudaStream_t st = nullptr;
  // side stream (lowest priority; st has the highest) for work that overlaps the
  // solver's main chain: the batched multishift's shift-field flushes
  cudaStream_t st2 = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t ev_fork[2] = {}, ev_join[2] = {};  // fork / join of st2 work, one pair per ring half

  // current links (trial::u) in FP64 and FP32
  double2* u64 = nullptr;
  float2* u32 = nullptr;
  bool links_ok = false;

  // staging for Fortran-layout host arrays (sized for one halo'd spinor)
  double2* stage = nullptr;
  size_t stage_elems = 0;
  double2* stage2 = nullptr;

  // FP64 work fields, one spinor each (4*V5 complex)
  std::vector<double2*> w64;
  // reduction scratch and device scalars
  double* partials = nullptr;
  size_t nparts = 0;         // entries of partials
  double* dscal = nullptr;   // general device scalar block
  int* iscal = nullptr;
  double* hscal = nullptr;   // pinned host mirror
  int* hiscal = nullptr;

  // named device buffers that grow on demand (solver workspaces, Phi0, dSdpi)
  enum Buf {
    B_X1 = 0,   // multishift outputs x1 (FP64), ndiag fields
    B_SF64,     // FP64 shift vectors
    B_OUT32,    // FP32 multishift outputs
    B_SF32,     // FP32 shift vectors
    B_WORK32,   // FP32 work vectors
    B_PHI0,     // qmrherm_module::Phi0 (FP64), ndiag fields
    B_DSDPI,    // gforce::dSdpi, [3][V3] FP64
    B_AUX,      // misc
    B_MD,       // MD spinors: Phi, X2, Xresult, R
    B_MDF,      // MD 3D fields: theta, thetat, pp (float) and dSdpi (double)
    B_HIST,     // batched multishift coefficient history
    B_RING,     // batched multishift residual ring
    B_COEF,     // batched multishift folded coefficients
    B_COUNT = 16
  };
  // rational approximations (remez.F90, remezg.F90): anum has n+1 entries
  struct Rational {
    bool set = false;
    int ndiag = 0, ndiagg = 0;
    std::vector<double> anum2, aden2, bnum2, bden2, anum4, aden4, bnum4, bden4;
    std::vector<double> anum2g, aden2g, bnum2g, bden2g, anum4g, aden4g, bnum4g, bden4g;
  } rat;
  // inverter residuals and the guidance-precision switch (params.F90:60-64)
  float rescga = 1e-8f, rescgg = 1e-6f;
  int spmd = 1;             // guidance solves: 0 FP64; 1 single precision (reference); 2, 3 mixed multishift
  int action_sp = 0;        // Hamiltonian and pseudofermion solves: 0 FP64; 2, 3 mixed multishift
  int max_qmr_iters = 50000;
  int ms_algo = 1;          // multishift: 0 = per-iteration shift updates, 1 = batched
  bool use_graphs = true;   // batched solver loops as one CUDA graph (WHILE node) per solve
  bool use_pdl = true;      // the batched multishift's and congrad's kernel chains as dependent launches (THR_PDL=0: off)
  // a batch of the batched FP64 multishift as one persistent kernel (msp.cu): 0 (default)
  // never; 1 where every stencil site block gets its own resident block; 2 wherever the
  // block shape allows (THR_CHAIN=0|1|2).  Off by default: on B200 the kernel chain with
  // dependent launches was as fast or faster at every lattice measured
  int chain_mode = 0;
  // cached batched-multishift graphs: FP64; FP32 vectors; FP32 and BF16 base
  // iteration with FP64 shift fields (the low-precision phase of the mixed solver)
  void* ms_graphs[4] = {};
  // mixed-precision multishift: relative base residual |r|/|input| below which the
  // base iteration leaves FP64 (FP32, BF16 storage); thr_set_mixed
  double mixed_switch[2] = {1e-8, 1e-13};
  int mixed_switched_at = 0;  // iteration the last mixed solve left FP64 at (0: never)
  void* cg_graph = nullptr;  // cached congrad graph
  // sweep directions of the solver kernels (THR_REVERSE=0|1|2): 0 all bottom up; 1 the
  // M^dagger-with-update stencil top down; 2 (default) directions alternate per iteration
  // so each kernel starts on the sites its predecessor wrote last
  int rev_sweep = 2;
  int overlap_flush = 1;     // batched multishift flushes on the side stream (THR_OVERLAP=0: in line)
  // measure_OWilson's coeffs(1:Ls) (prepZolo) and their device copy
  std::vector<double> zolo;
  double* zolo_dev = nullptr;
  bool zolo_dirty = false;
  double md_counts[8] = {};  // ancg, ancgpv, ancgf, ancgfpv, ancgh, ancghpv, ancgpf, ancgpfpv
  // One leapfrog step of evolve_theta_pp as a CUDA graph (md.cu).  While it is
  // captured (md_capture), the solver code adds its batch loops as WHILE nodes of
  // the captured graph (their bodies captured on st3), takes each multishift's
  // initial state from its own pinned template (ms_tmpl, a slot per solve of the
  // step), counts iterations on the device (md_dev: per-counter sums, the OR of
  // the solves' status and the step's exit draw) and never synchronises; a
  // buffer that would have to grow makes the capture fail (the step then runs
  // host-driven).  THR_MD_GRAPH=0 turns the graph off.
  bool md_capture = false;
  bool use_md_graph = true;
  cudaStream_t st3 = nullptr;
  void* ms_tmpl = nullptr;  // pinned, kMsTemplates MsState slots
  int ms_tmpl_next = 0;
  void* md_graph = nullptr;  // cached step graph (md.cu)
  unsigned long long buf_gen = 0;  // bumped whenever a device buffer is (re)allocated
  void* bufs[B_COUNT] = {};
  size_t buf_bytes[B_COUNT] = {};
  bool phi0_valid = false;
  thr::Rng rng;  // random's module state
  int buffer(int id, size_t bytes, void** out);  // contents preserved only if not regrown

  // optional per-kernel timing: CUDA events around selected launches
  // kernel timing: every prof_stride-th launch of each kind is bracketed by events
  // (P_DSLASH_LOW / P_DSLASH_DAG_LOW: the same stencils in the low-precision phase of the mixed multishift;
  // P_ALPHA, P_LAMBDA: the batched multishift's one-block scalar steps k_alpha and k_lambda)
  enum ProfKernel {
    P_DSLASH = 0, P_SHIFTUPD = 1, P_DSLASH_DAG = 2, P_DSLASH_LOW = 3, P_DSLASH_DAG_LOW = 4, P_ALPHA = 5, P_LAMBDA = 6,
    P_COUNT = 7
  };
  bool prof_on = false;
  int prof_stride = 1;
  long long prof_seen[P_COUNT] = {};         // launches offered to prof_begin
  double prof_work[P_COUNT] = {};            // launches that did work (guarded launches excluded)
  std::vector<cudaEvent_t> prof_ev;          // pairs
  std::vector<int> prof_kind;                // -1: dropped (a launch that skipped its work)
  std::vector<double> prof_bytes;            // algorithmic bytes of the sampled launch
  std::vector<long long> prof_tag;           // iteration of the sampled launch within its solve
  // events go on stream `on` (nullptr: st)
  int prof_begin(int kind, double bytes, long long tag = -1, cudaStream_t on = nullptr);  // pair index or -1
  void prof_end(int idx, cudaStream_t on = nullptr);
  void prof_set_bytes(int idx, double bytes);
  // drop the sampled launches since entry `first` whose tag is >= iters (skipped work)
  void prof_trim(size_t first, long long iters);

  size_t n4() const { return (size_t)g.v5 * 4; }  // complex elements of one spinor
  size_t nf5() const { return (size_t)(g.ls + 2) * (g.lx + 2) * (g.ly + 2) * (g.lt + 2) * 4; }
  size_t nfl() const { return (size_t)(g.lx + 2) * (g.ly + 2) * (g.lt + 2) * 3; }

  int ensure_w64(int count);
  int upload_spinor(double2* dst, const double* host);     // Fortran halo'd -> device
  int download_spinor(double* host, const double2* src);   // device -> Fortran halo'd
  int use_links(const double* u_host);                    // NULL keeps current links
  int coef_dev(const float* theta_dev);                   // gauge.F90 coef on device theta
  int sync();
};
