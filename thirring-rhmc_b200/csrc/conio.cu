// conio.cu -- configuration checkpoints (dwf3d_lib.F90:618-767): the `con`
// file with theta and the generator seed, and the `random_seed` text file.
//
// Two byte layouts exist for the same content (theta: real(Lx,Ly,Lt,3) in
// Fortran order, seed: real(dp)):
//   THR_CON_SERIAL  the serial build's unformatted sequential record
//                   (dwf3d_lib.F90:651-653, :711-714):
//                   [int32 12V+8][theta, 12V bytes][seed][int32 12V+8]
//   THR_CON_MPIIO   the MPI build (:632-649, :683-704): theta written by
//                   MPI-IO at offset 0, then the seed and the record length
//                   written at offset 12V+4 by a stream-access unit, which
//                   leaves bytes 12V..12V+3 as whatever the file held there
//                   (zero for a new file).
// Reading detects the layout from the leading record marker.  V = Lx*Ly*Lt.
// Host code only: nothing here touches the GPU.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/thirring_b200.h"

namespace {

bool read_all(const char* path, std::vector<unsigned char>& buf) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  unsigned char tmp[1 << 16];
  size_t n;
  while ((n = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + n);
  std::fclose(f);
  return true;
}

int32_t rd_i32(const unsigned char* p) {
  int32_t v;
  std::memcpy(&v, p, 4);
  return v;
}

}  // namespace

extern "C" {

int thr_read_con(const char* path, int lx, int ly, int lt, float* theta, double* seed, int* format) {
  if (!path || !theta || !seed || lx < 1 || ly < 1 || lt < 1) return THR_ERR_BADARG;
  const size_t nth = 3 * (size_t)lx * ly * lt;
  const size_t rec = 4 * nth + 8;
  std::vector<unsigned char> b;
  if (!read_all(path, b)) return THR_ERR_BADARG;
  if (b.size() >= rec + 8 && (size_t)rd_i32(b.data()) == rec && (size_t)rd_i32(b.data() + 4 + rec) == rec) {
    std::memcpy(theta, b.data() + 4, 4 * nth);
    std::memcpy(seed, b.data() + 4 + 4 * nth, 8);
    if (format) *format = THR_CON_SERIAL;
    return THR_OK;
  }
  if (b.size() >= 4 * nth + 12 && (size_t)rd_i32(b.data() + 4 * nth + 12) == rec) {
    std::memcpy(theta, b.data(), 4 * nth);
    std::memcpy(seed, b.data() + 4 * nth + 4, 8);
    if (format) *format = THR_CON_MPIIO;
    return THR_OK;
  }
  return THR_ERR_BADSHAPE;  // not a configuration of this lattice size
}

int thr_write_con(const char* path, int lx, int ly, int lt, const float* theta, double seed, int format) {
  if (!path || !theta || lx < 1 || ly < 1 || lt < 1) return THR_ERR_BADARG;
  if (format != THR_CON_SERIAL && format != THR_CON_MPIIO) return THR_ERR_BADARG;
  const size_t nth = 3 * (size_t)lx * ly * lt;
  const int32_t rec = (int32_t)(4 * nth + 8);
  FILE* f = std::fopen(path, "wb");
  if (!f) return THR_ERR_BADARG;
  bool ok = true;
  const int32_t zero = 0;
  if (format == THR_CON_SERIAL) {
    ok = std::fwrite(&rec, 4, 1, f) == 1 && std::fwrite(theta, 4, nth, f) == nth && std::fwrite(&seed, 8, 1, f) == 1 &&
         std::fwrite(&rec, 4, 1, f) == 1;
  } else {
    ok = std::fwrite(theta, 4, nth, f) == nth && std::fwrite(&zero, 4, 1, f) == 1 && std::fwrite(&seed, 8, 1, f) == 1 &&
         std::fwrite(&rec, 4, 1, f) == 1;
  }
  ok = (std::fclose(f) == 0) && ok;
  return ok ? THR_OK : THR_ERR_BADARG;
}

// readseed / saveseed (dwf3d_lib.F90:719-767): one list-directed real(dp)
int thr_readseed(const char* path, double* seed) {
  if (!path || !seed) return THR_ERR_BADARG;
  FILE* f = std::fopen(path, "r");
  if (!f) return THR_ERR_BADARG;
  double v;
  const int n = std::fscanf(f, "%lf", &v);
  std::fclose(f);
  if (n != 1) return THR_ERR_BADARG;
  *seed = v;
  return THR_OK;
}

int thr_saveseed(const char* path, double seed) {
  if (!path) return THR_ERR_BADARG;
  FILE* f = std::fopen(path, "w");
  if (!f) return THR_ERR_BADARG;
  // list-directed output of a real(dp): the value in fixed notation, exact for
  // the integer-valued seeds the generator holds (below 2^48)
  const int n = (std::fabs(seed) < 1e17 && seed == std::floor(seed)) ? std::fprintf(f, "   %.4f     \n", seed)
                                                                       : std::fprintf(f, "   %.17g\n", seed);
  const bool ok = (std::fclose(f) == 0) && n > 0;
  return ok ? THR_OK : THR_ERR_BADARG;
}

}  // extern "C"
