// Histogram bins as sinc records: a tile of SE_TILE bins of one element pair becomes records
// (r_k = (k + 0.5) bin, weight n_k); empty bins carry no weight (the reference skips them,
// CalcFunctions.cpp:857).  Used by the histogram -> I(q) transform.
#pragma once
#include "sinc_engine.cuh"

namespace xns_sinc {

struct BinSrc {
  const unsigned long long *hist;
  uint32_t nhist;
  uint32_t tiles_per_pair;
  double bin;

  __device__ uint32_t cls(unsigned long long w) const { return (uint32_t)(w / tiles_per_pair); }

  __device__ int fill(unsigned long long w, PairRec *pr, void *, const SincParams &p, uint32_t cls) const {
    const uint32_t t = (uint32_t)(w / tiles_per_pair);
    const uint32_t b0 = (uint32_t)(w % tiles_per_pair) * SE_TILE;
    const unsigned long long *h = hist + (size_t)t * nhist;
    for (int e = threadIdx.x; e < SE_TILE; e += SE_THREADS) {
      const uint32_t k = b0 + e;
      PairRec rec = null_rec();
      if (k < nhist) {
        unsigned long long n = h[k];
        if (n) rec = make_rec(p, cls, ((double)k + 0.5) * bin, (double)n);
      }
      pr[e] = rec;
    }
    __syncthreads();
    return SE_TILE;
  }
};

}  // namespace xns_sinc
