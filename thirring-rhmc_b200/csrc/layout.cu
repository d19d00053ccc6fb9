// layout.cu -- gather/scatter between the reference's Fortran arrays (with
// one-site halos, column-major) and the device fields.  The Fortran array is
// first copied verbatim into a device staging buffer; these kernels then
// gather its interior (inputs; halos are ignored because the device uses
// periodic indexing) or write the interior plus the periodic images into
// every halo position (outputs), which is what the reference's halo update
// (comms5.F90:135-194 on a 1x1x1x1 grid) leaves there.
#include "thr_common.cuh"
#include "thr_kernels.h"

namespace thr {

namespace {
__device__ __forceinline__ int wrap(int c, int l) { return c < 0 ? c + l : (c >= l ? c - l : c); }

__device__ __forceinline__ size_t f5(const Geom& g, int s, int x, int y, int t, int d) {
  // 0-based interior coordinates -> offset in (0:Ls+1,0:Lx+1,0:Ly+1,0:Lt+1,4)
  return (size_t)(s + 1) +
         (size_t)(g.ls + 2) * ((size_t)(x + 1) + (size_t)(g.lx + 2) * ((size_t)(y + 1) + (size_t)(g.ly + 2) * ((size_t)(t + 1) + (size_t)(g.lt + 2) * d)));
}

template <class S>
__global__ void k_from_fortran_spinor(S* out, const double2* fin, Geom g) {
  size_t n = (size_t)g.v5 * 4;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    int s = (int)(i % g.ls);
    size_t r = i / g.ls;
    int site = (int)(r % g.v3);
    int d = (int)(r / g.v3);
    int x, y, t;
    site_coords(g, site, x, y, t);
    double2 v = fin[f5(g, s, x, y, t, d)];
    Sto<S>::st(out, i, typename Sto<S>::C{(typename Sto<S>::R)v.x, (typename Sto<S>::R)v.y});
  }
}

__global__ void k_to_fortran_spinor(double2* fout, const double2* in, Geom g) {
  // every element of the halo'd array, interior and halos, gets its periodic image
  const int LS2 = g.ls + 2, LX2 = g.lx + 2, LY2 = g.ly + 2, LT2 = g.lt + 2;
  size_t n = (size_t)LS2 * LX2 * LY2 * LT2 * 4;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    size_t r = i;
    int s = (int)(r % LS2); r /= LS2;
    int x = (int)(r % LX2); r /= LX2;
    int y = (int)(r % LY2); r /= LY2;
    int t = (int)(r % LT2);
    int d = (int)(r / LT2);
    int ss = wrap(s - 1, g.ls), xx = wrap(x - 1, g.lx), yy = wrap(y - 1, g.ly), tt = wrap(t - 1, g.lt);
    fout[i] = in[sidx(g, ss, site_index(g, xx, yy, tt), d)];
  }
}

__global__ void k_to_fortran_noh(double2* fout, const double2* in, Geom g) {
  size_t n = (size_t)g.v5 * 4;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    size_t r = i;
    int s = (int)(r % g.ls); r /= g.ls;
    int x = (int)(r % g.lx); r /= g.lx;
    int y = (int)(r % g.ly); r /= g.ly;
    int t = (int)(r % g.lt);
    int d = (int)(r / g.lt);
    fout[i] = in[sidx(g, s, site_index(g, x, y, t), d)];
  }
}

__global__ void k_from_fortran_noh(double2* out, const double2* fin, Geom g) {
  size_t n = (size_t)g.v5 * 4;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    size_t r = i;
    int s = (int)(r % g.ls); r /= g.ls;
    int x = (int)(r % g.lx); r /= g.lx;
    int y = (int)(r % g.ly); r /= g.ly;
    int t = (int)(r % g.lt);
    int d = (int)(r / g.lt);
    out[sidx(g, s, site_index(g, x, y, t), d)] = fin[i];
  }
}

__global__ void k_from_fortran_links(double2* out, const double2* fin, Geom g) {
  int n = g.v3 * 3;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int site = i % g.v3, mu = i / g.v3;
    int x, y, t;
    site_coords(g, site, x, y, t);
    out[i] = fin[(x + 1) + (size_t)(g.lx + 2) * ((y + 1) + (size_t)(g.ly + 2) * ((t + 1) + (size_t)(g.lt + 2) * mu))];
  }
}

__global__ void k_to_fortran_links(double2* fout, const double2* in, Geom g) {
  const int LX2 = g.lx + 2, LY2 = g.ly + 2, LT2 = g.lt + 2;
  int n = LX2 * LY2 * LT2 * 3;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int r = i;
    int x = r % LX2; r /= LX2;
    int y = r % LY2; r /= LY2;
    int t = r % LT2;
    int mu = r / LT2;
    fout[i] = in[(size_t)mu * g.v3 + site_index(g, wrap(x - 1, g.lx), wrap(y - 1, g.ly), wrap(t - 1, g.lt))];
  }
}

template <class T>
__global__ void k_from_fortran_3(T* out, const T* fin, Geom g) {
  int n = g.v3 * 3;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int r = i;
    int x = r % g.lx; r /= g.lx;
    int y = r % g.ly; r /= g.ly;
    int t = r % g.lt;
    int mu = r / g.lt;
    out[(size_t)mu * g.v3 + site_index(g, x, y, t)] = fin[i];
  }
}
template <class T>
__global__ void k_to_fortran_3(T* fout, const T* in, Geom g) {
  int n = g.v3 * 3;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int r = i;
    int x = r % g.lx; r /= g.lx;
    int y = r % g.ly; r /= g.ly;
    int t = r % g.lt;
    int mu = r / g.lt;
    fout[i] = in[(size_t)mu * g.v3 + site_index(g, x, y, t)];
  }
}

__global__ void k_to_fortran_ps(float* fout, const float* in, Geom g) {
  const int LX2 = g.lx + 2, LY2 = g.ly + 2, LT2 = g.lt + 2;
  int n = LX2 * LY2 * LT2 * 2;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int r = i;
    int x = r % LX2; r /= LX2;
    int y = r % LY2; r /= LY2;
    int t = r % LT2;
    int c = r / LT2;
    fout[i] = in[(size_t)c * g.v3 + site_index(g, wrap(x - 1, g.lx), wrap(y - 1, g.ly), wrap(t - 1, g.lt))];
  }
}

inline unsigned grid_for(size_t n, int threads = 256) {
  size_t b = (n + threads - 1) / threads;
  if (b > device_sms() * 32) b = device_sms() * 32;
  if (b < 1) b = 1;
  return (unsigned)b;
}
}  // namespace

template <class S>
void from_fortran_spinor(const Geom& g, S* out, const double2* fin, cudaStream_t st) {
  k_from_fortran_spinor<S><<<grid_for((size_t)g.v5 * 4), 256, 0, st>>>(out, fin, g);
}
template void from_fortran_spinor<double2>(const Geom&, double2*, const double2*, cudaStream_t);
template void from_fortran_spinor<float2>(const Geom&, float2*, const double2*, cudaStream_t);

void to_fortran_spinor(const Geom& g, double2* fout, const double2* in, cudaStream_t st) {
  size_t n = (size_t)(g.ls + 2) * (g.lx + 2) * (g.ly + 2) * (g.lt + 2) * 4;
  k_to_fortran_spinor<<<grid_for(n), 256, 0, st>>>(fout, in, g);
}
void to_fortran_noh(const Geom& g, double2* fout, const double2* in, cudaStream_t st) {
  k_to_fortran_noh<<<grid_for((size_t)g.v5 * 4), 256, 0, st>>>(fout, in, g);
}
void from_fortran_noh(const Geom& g, double2* out, const double2* fin, cudaStream_t st) {
  k_from_fortran_noh<<<grid_for((size_t)g.v5 * 4), 256, 0, st>>>(out, fin, g);
}
void from_fortran_links(const Geom& g, double2* out, const double2* fin, cudaStream_t st) {
  k_from_fortran_links<<<grid_for((size_t)g.v3 * 3), 256, 0, st>>>(out, fin, g);
}
void to_fortran_links(const Geom& g, double2* fout, const double2* in, cudaStream_t st) {
  size_t n = (size_t)(g.lx + 2) * (g.ly + 2) * (g.lt + 2) * 3;
  k_to_fortran_links<<<grid_for(n), 256, 0, st>>>(fout, in, g);
}
void from_fortran_f3(const Geom& g, float* out, const float* fin, cudaStream_t st) {
  k_from_fortran_3<float><<<grid_for((size_t)g.v3 * 3), 256, 0, st>>>(out, fin, g);
}
void to_fortran_f3(const Geom& g, float* fout, const float* in, cudaStream_t st) {
  k_to_fortran_3<float><<<grid_for((size_t)g.v3 * 3), 256, 0, st>>>(fout, in, g);
}
void from_fortran_d3(const Geom& g, double* out, const double* fin, cudaStream_t st) {
  k_from_fortran_3<double><<<grid_for((size_t)g.v3 * 3), 256, 0, st>>>(out, fin, g);
}
void to_fortran_d3(const Geom& g, double* fout, const double* in, cudaStream_t st) {
  k_to_fortran_3<double><<<grid_for((size_t)g.v3 * 3), 256, 0, st>>>(fout, in, g);
}
void to_fortran_ps(const Geom& g, float* fout, const float* in, cudaStream_t st) {
  size_t n = (size_t)(g.lx + 2) * (g.ly + 2) * (g.lt + 2) * 2;
  k_to_fortran_ps<<<grid_for(n), 256, 0, st>>>(fout, in, g);
}

}  // namespace thr
