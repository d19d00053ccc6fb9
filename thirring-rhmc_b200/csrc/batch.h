// batch.h -- many right-hand sides or many lattices in one launch.
//
// A batch is a table of entries; entry e is a spinor field of geometry g at
// element offset `off` of a packed array, with links at element offset
// `uoff` of a packed link array (0 for every entry when the entries are
// right-hand sides on one lattice).  The stencil's work is cut into blocks
// of 256 threads (spb sites of Ls threads each); blk0 is the entry's first
// work block in the global numbering, so one persistent launch walks the
// work of all entries whatever their sizes.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "thr_common.cuh"

namespace thr {

struct BatchEntry {
  Geom g;
  long long off;   // element offset of the entry's spinor in packed fields
  long long uoff;  // element offset of the entry's links
  int blk0;        // first work block
  int spb;         // sites per work block
  int nblk;        // work blocks of this entry
  int pad;
};

struct BatchTable {
  int nent = 0;
  int total_blocks = 0;
  long long total_elems = 0;  // sum of 4*V5 over entries
  long long total_links = 0;  // sum of 3*V3 over distinct link sets
  std::vector<BatchEntry> host;
  BatchEntry* dev = nullptr;
  ~BatchTable();
  // shared_links: all entries use the links at offset 0 (right-hand sides of one lattice)
  int build(const std::vector<Geom>& geoms, bool shared_links, cudaStream_t st);
};

template <class S>
int launch_dslash_batch(const BatchTable& b, int kernel, bool dag, S* out, const S* in, const typename Sto<S>::C* u,
                        float am, int imass, float am3, cudaStream_t st, const int* skip, const S* aux,
                        double* partials, int grid = 0);
// the batch stencil with a CG epilogue: epi 2 out = M in with a partial of |out|^2 per work
// block; epi 4 rv -= coef[e * coef_stride] (M in) in place (arithmetic type, out unused)
// with a partial of |rv|^2 per work block
template <class S>
int launch_dslash_batch_fused(const BatchTable& b, int kernel, bool dag, int epi, S* out, const S* in,
                              const typename Sto<S>::C* u, float am, int imass, float am3, cudaStream_t st,
                              const int* skip, typename Sto<S>::C* rv, const double* coef, int coef_stride,
                              double* partials, int grid = 0);

}  // namespace thr
