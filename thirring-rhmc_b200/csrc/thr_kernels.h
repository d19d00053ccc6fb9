// thr_kernels.h -- launchers shared between the translation units of the
// CUDA library.  Host-callable, stream-ordered, no allocation.
#pragma once
#include <utility>

#include "thr_common.cuh"

namespace thr {

// number of per-block partial sums a reduction may write (>= any grid used)
constexpr int kMaxPartials = 4096;

// Launches kern<<<grid, block, smem, st>>>(args...); with pdl as a programmatic dependent of
// the previous kernel on st (the kernel must call pdl_wait() before it reads that kernel's
// results), so that its launch and scheduling overlap the predecessor's tail.
template <typename... KArgs, typename... Args>
inline void launch_k(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, bool pdl,
                     Args&&... args) {
  if (!pdl) {
    kern<<<grid, block, smem, st>>>(std::forward<Args>(args)...);
    return;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// streaming multiprocessors of the current device (looked up once per device);
// grid-stride kernels size their grids as a multiple of it
int device_sms();

dim3 stencil_block(const Geom& g, int kernel);
unsigned stencil_grid(const Geom& g, int kernel);  // blocks of one stencil launch (= partials it writes)
// partials an epilogue launch writes (the FP64 Shamir kernel on staged tiles has its own grid)
unsigned stencil_parts(const Geom& g, int kernel, bool fp64);

// dslash.cu
template <class S>
int launch_dslash(const Geom& g, int kernel, bool dag, S* out, const S* in, const typename Sto<S>::C* u, float am,
                  int imass, float am3, cudaStream_t st, const int* skip = nullptr);
// as launch_dslash, but never runs the autotuner's timing launches (no events, no
// synchronisation): the register budget is one tuned earlier in the process or the
// default, which gives the same results
template <class S>
int launch_dslash_untuned(const Geom& g, int kernel, bool dag, S* out, const S* in, const typename Sto<S>::C* u,
                          float am, int imass, float am3, cudaStream_t st, const int* skip = nullptr);
// rnew = rold + (*coef) * (M or M^dagger) in, without storing the stencil's output,
// and one FP64 partial per block of |rnew|^2.  rev != 0: blocks take the sites from
// the top down (same results; better L2 reuse of a field written just before)
template <class S>
int launch_dslash_axpy(const Geom& g, int kernel, bool dag, S* rnew, const S* in, const typename Sto<S>::C* u,
                       float am, int imass, float am3, cudaStream_t st, const int* skip, const S* rold,
                       const double* coef, double* partials, int rev = 0, bool pdl = false);
// same, with one FP64 partial per block of sum |out|^2
template <class S>
int launch_dslash_norm(const Geom& g, int kernel, bool dag, S* out, const S* in, const typename Sto<S>::C* u,
                       float am, int imass, float am3, cudaStream_t st, const int* skip, double* partials,
                       int rev = 0, bool pdl = false);

// odslash / odslashd (measure_OWilson.F90:14-167), FP64, with the slice coefficients zc[0..Ls-1] on the device
int launch_odslash(const Geom& g, bool dag, double2* out, const double2* in, const double2* u, float am, int imass,
                   float am3, const double* zc, cudaStream_t st, const int* skip = nullptr);

// hnew = (M or M^dagger) in + (*coef) * hold and one FP64 partial per block of |hnew|^2
// (hnew and hold distinct fields)
template <class S>
int launch_dslash_accum(const Geom& g, int kernel, bool dag, S* hnew, const S* in, const typename Sto<S>::C* u,
                        float am, int imass, float am3, cudaStream_t st, const int* skip, const S* hold,
                        const double* coef, double* partials, int rev = 0, bool pdl = false);

// layout.cu: Fortran halo'd host layout <-> device fields
// spinor (0:Ls+1,0:Lx+1,0:Ly+1,0:Lt+1,4) complex(dp)  <-> S[4][V3][Ls]
template <class S>
void from_fortran_spinor(const Geom& g, S* out, const double2* fin, cudaStream_t st);
void to_fortran_spinor(const Geom& g, double2* fout, const double2* in, cudaStream_t st);
// shift outputs (Ls,Lx,Ly,Lt,4) per shift, no halo
void to_fortran_noh(const Geom& g, double2* fout, const double2* in, cudaStream_t st);
void from_fortran_noh(const Geom& g, double2* out, const double2* fin, cudaStream_t st);
// links (0:Lx+1,0:Ly+1,0:Lt+1,3) complex(dp) <-> double2[3][V3]
void from_fortran_links(const Geom& g, double2* out, const double2* fin, cudaStream_t st);
void to_fortran_links(const Geom& g, double2* fout, const double2* in, cudaStream_t st);
// (Lx,Ly,Lt,3) real or real(dp) <-> [3][V3]
void from_fortran_f3(const Geom& g, float* out, const float* fin, cudaStream_t st);
void to_fortran_f3(const Geom& g, float* fout, const float* in, cudaStream_t st);
void from_fortran_d3(const Geom& g, double* out, const double* fin, cudaStream_t st);
void to_fortran_d3(const Geom& g, double* fout, const double* in, cudaStream_t st);
// ps (0:Lx+1,0:Ly+1,0:Lt+1,2) real from device [2][V3] (halo = periodic images)
void to_fortran_ps(const Geom& g, float* fout, const float* in, cudaStream_t st);

// blas.cu
template <class Sd, class Ss>
void convert(Sd* dst, const Ss* src, size_t n, cudaStream_t st);
void links_to_float(float2* dst, const double2* src, size_t n, cudaStream_t st);
// per-block partial sums of sum |a|^2 (FP64 accumulation); returns #blocks written
template <class S>
int norm2_partials(const S* a, size_t n, double* partials, cudaStream_t st);
template <class S>
int redot_partials(const S* a, const S* b, size_t n, double* partials, cudaStream_t st);
// out = sum of partials (single block, fixed order)
void finish_sum(const double* partials, int nparts, double* out, cudaStream_t st);
// y = a*x + y / y = x + a*y etc. with device or host scalars
void axpy_d(double2* y, const double2* x, double a, size_t n, cudaStream_t st);
void scale_copy_d(double2* y, const double2* x, double a, size_t n, cudaStream_t st);  // y = a*x

}  // namespace thr
