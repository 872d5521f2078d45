// Pair-distance histogram (replaces calcHist, CalcFunctions.cpp:757-809, and calcHistKernel,
// CalcFunctionsCUDA.cu:814-920).
//
// Counts are bit-identical to the reference's (exact FP64 bin decision, hist_bin.cuh).  At the
// reference's 0.001 A bins a 2e5-atom structure has ~3e5 bins per element pair: far more than a shared
// memory histogram holds, and one global atomic per pair leaves the kernel bound by L2 atomics.  So
// the pairs are ordered by distance first:
//   1. atoms of each element are counting-sorted into cubic cells of ~CELL_TARGET atoms
//      (cell_count / cell_scan / cell_scatter kernels); each cell is cut into tiles of <= 64 atoms
//      with a bounding box (tile_build / tile_bbox);
//   2. every tile pair (upper triangle within an element, all pairs across elements) gets the bin
//      range [kmin, kmax] its bounding boxes allow, and is counting-sorted by (element pair,
//      kmin / BUCKET) (pair_key / key_scan / pair_scatter);
//   3. hist_window_kernel: one CTA per SM walks a contiguous run of that list, one tile pair per warp,
//      and counts into a WIN-bin u32 window of shared memory that slides up the distance axis (bins
//      that leave the window are added to the u64 global histogram once per CTA);
//   4. hist_wide_kernel: tile pairs whose range is wider than the window (sparse elements) count
//      straight into the global histogram.
// Atom order inside a cell and list order inside a bucket come from atomics, but counts do not depend
// on either.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cmath>

#include "hist_bin.cuh"
#include "schedule.cuh"

using namespace xns_hist;

namespace {

constexpr int CELL_TARGET = 56;      // mean atoms per cell over an element's bounding box
constexpr int TILE_MAX = 64;         // atoms per tile
constexpr int MAX_CELLS_AXIS = 256;
constexpr int HW_WARPS = 16;
constexpr int HW_THREADS = 32 * HW_WARPS;
constexpr uint32_t WIN = 50 * 1024;  // window bins
constexpr uint32_t BUCKET = 1024;    // distance bucket of the tile-pair sort, in bins
constexpr int SCAN_THREADS = 1024;

struct Tile {
  uint32_t start, count, elem, pad;
  double lo[3], hi[3];
};
struct TilePair {
  uint32_t I, J, kmin, kmax;
};
struct ElemGrid {
  double o[3], inv[3];
  uint32_t n[3];
  uint32_t base;  // first cell of this element
  uint32_t atom0, natoms;
};
struct CtaRange {
  uint32_t begin, end, type, pad;
};

// doubles -> u64 keys with the same order, for atomicMin / atomicMax
__device__ __forceinline__ unsigned long long ord_key(double x) {
  unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
double ord_value(unsigned long long u) {
  unsigned long long b = (u >> 63) ? (u & 0x7fffffffffffffffull) : ~u;
  double x;
  memcpy(&x, &b, sizeof x);
  return x;
}

__global__ void elem_bbox_kernel(const double *__restrict__ X, const double *__restrict__ Y, const double *__restrict__ Z,
                                 const ElemGrid *__restrict__ eg, unsigned long long *__restrict__ bmin,
                                 unsigned long long *__restrict__ bmax) {
  const int e = blockIdx.y;
  const uint32_t a0 = eg[e].atom0, a1 = a0 + eg[e].natoms;
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t i = a0 + blockIdx.x * blockDim.x + threadIdx.x; i < a1; i += gridDim.x * blockDim.x) {
    const double v[3] = {X[i], Y[i], Z[i]};
    for (int k = 0; k < 3; k++) {
      mn[k] = fmin(mn[k], v[k]);
      mx[k] = fmax(mx[k], v[k]);
    }
  }
  for (int k = 0; k < 3; k++)
    for (int o = 16; o; o >>= 1) {
      mn[k] = fmin(mn[k], __shfl_down_sync(0xffffffffu, mn[k], o));
      mx[k] = fmax(mx[k], __shfl_down_sync(0xffffffffu, mx[k], o));
    }
  if ((threadIdx.x & 31) == 0 && a1 > a0)
    for (int k = 0; k < 3; k++) {
      atomicMin(bmin + 3 * e + k, ord_key(mn[k]));
      atomicMax(bmax + 3 * e + k, ord_key(mx[k]));
    }
}

__device__ __forceinline__ uint32_t cell_of(const ElemGrid &g, double x, double y, double z) {
  const double v[3] = {x, y, z};
  uint32_t c[3];
  for (int k = 0; k < 3; k++) {
    double f = (v[k] - g.o[k]) * g.inv[k];
    int ci = (int)f;
    c[k] = (uint32_t)min(max(ci, 0), (int)g.n[k] - 1);
  }
  return g.base + (c[2] * g.n[1] + c[1]) * g.n[0] + c[0];
}

__global__ void cell_count_kernel(const double *__restrict__ X, const double *__restrict__ Y, const double *__restrict__ Z,
                                  const ElemGrid *__restrict__ eg, uint32_t *__restrict__ cid, uint32_t *__restrict__ cnt) {
  const ElemGrid g = eg[blockIdx.y];
  for (uint32_t i = g.atom0 + blockIdx.x * blockDim.x + threadIdx.x; i < g.atom0 + g.natoms; i += gridDim.x * blockDim.x) {
    const uint32_t c = cell_of(g, X[i], Y[i], Z[i]);
    cid[i] = c;
    atomicAdd(cnt + c, 1u);
  }
}

// Single-CTA exclusive scan of up to two u32 sequences (a and, if b_out, the tile counts derived from
// a): each thread scans a contiguous chunk, the chunk totals are scanned in shared memory.
__global__ void __launch_bounds__(SCAN_THREADS) scan_kernel(const uint32_t *__restrict__ a, uint32_t n,
                                                            uint32_t *__restrict__ a_out, uint32_t *__restrict__ b_out,
                                                            uint32_t *__restrict__ totals) {
  __shared__ uint32_t sa[SCAN_THREADS], sb[SCAN_THREADS];
  const uint32_t per = (n + SCAN_THREADS - 1) / SCAN_THREADS;
  const uint32_t lo = min(n, threadIdx.x * per), hi = min(n, lo + per);
  uint32_t ta = 0, tb = 0;
  for (uint32_t i = lo; i < hi; i++) {
    ta += a[i];
    tb += (a[i] + TILE_MAX - 1) / TILE_MAX;
  }
  sa[threadIdx.x] = ta;
  sb[threadIdx.x] = tb;
  __syncthreads();
  for (int o = 1; o < SCAN_THREADS; o <<= 1) {  // Hillis-Steele inclusive scan
    uint32_t va = threadIdx.x >= o ? sa[threadIdx.x - o] : 0, vb = threadIdx.x >= o ? sb[threadIdx.x - o] : 0;
    __syncthreads();
    sa[threadIdx.x] += va;
    sb[threadIdx.x] += vb;
    __syncthreads();
  }
  uint32_t pa = sa[threadIdx.x] - ta, pb = sb[threadIdx.x] - tb;
  for (uint32_t i = lo; i < hi; i++) {
    a_out[i] = pa;
    pa += a[i];
    if (b_out) {
      b_out[i] = pb;
      pb += (a[i] + TILE_MAX - 1) / TILE_MAX;
    }
  }
  if (threadIdx.x == SCAN_THREADS - 1) {
    totals[0] = sa[SCAN_THREADS - 1];
    totals[1] = sb[SCAN_THREADS - 1];
  }
}

__global__ void cell_scatter_kernel(const double *__restrict__ X, const double *__restrict__ Y, const double *__restrict__ Z,
                                    uint32_t n, const uint32_t *__restrict__ cid, const uint32_t *__restrict__ cell_off,
                                    uint32_t *__restrict__ cursor, double *__restrict__ Xs, double *__restrict__ Ys,
                                    double *__restrict__ Zs) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t c = cid[i];
    const uint32_t p = cell_off[c] + atomicAdd(cursor + c, 1u);
    Xs[p] = X[i];
    Ys[p] = Y[i];
    Zs[p] = Z[i];
  }
}

// Cells -> tiles: a cell of n atoms becomes ceil(n/64) tiles of near-equal size.
__global__ void tile_build_kernel(const uint32_t *__restrict__ cnt, const uint32_t *__restrict__ cell_off,
                                  const uint32_t *__restrict__ tile_off, uint32_t ncells, const ElemGrid *__restrict__ eg,
                                  uint32_t nel, Tile *__restrict__ tiles) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells; c += gridDim.x * blockDim.x) {
    const uint32_t n = cnt[c];
    if (!n) continue;
    uint32_t e = 0;
    while (e + 1 < nel && c >= eg[e + 1].base) e++;
    const uint32_t nt = (n + TILE_MAX - 1) / TILE_MAX;
    uint32_t s = cell_off[c];
    for (uint32_t t = 0; t < nt; t++) {
      const uint32_t cnt_t = n / nt + (t < n % nt ? 1 : 0);
      Tile tl;
      tl.start = s;
      tl.count = cnt_t;
      tl.elem = e;
      tl.pad = 0;
      tiles[tile_off[c] + t] = tl;
      s += cnt_t;
    }
  }
}

__global__ void tile_bbox_kernel(const double *__restrict__ X, const double *__restrict__ Y, const double *__restrict__ Z,
                                 Tile *__restrict__ tiles, uint32_t ntiles) {
  const uint32_t lane = threadIdx.x & 31;
  for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntiles; t += (gridDim.x * blockDim.x) >> 5) {
    const uint32_t s = tiles[t].start, n = tiles[t].count;
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = lane; i < n; i += 32) {
      const double v[3] = {X[s + i], Y[s + i], Z[s + i]};
      for (int k = 0; k < 3; k++) {
        mn[k] = fmin(mn[k], v[k]);
        mx[k] = fmax(mx[k], v[k]);
      }
    }
    for (int k = 0; k < 3; k++)
      for (int o = 16; o; o >>= 1) {
        mn[k] = fmin(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
        mx[k] = fmax(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
      }
    if (lane < 3) {
      tiles[t].lo[lane] = mn[lane];
      tiles[t].hi[lane] = mx[lane];
    }
  }
}

// Bin range of all pairs between two tiles, widened by 2 bins against rounding.
__device__ __forceinline__ void tile_pair_range(const Tile &A, const Tile &B, double inv_bin, uint32_t *kmin, uint32_t *kmax) {
  double g2 = 0, s2 = 0;
  for (int k = 0; k < 3; k++) {
    const double g = fmax(0.0, fmax(B.lo[k] - A.hi[k], A.lo[k] - B.hi[k]));
    const double s = fmax(B.hi[k] - A.lo[k], A.hi[k] - B.lo[k]);
    g2 += g * g;
    s2 += s * s;
  }
  const double lo = floor(sqrt(g2) * inv_bin) - 2.0, hi = floor(sqrt(s2) * inv_bin) + 2.0;
  *kmin = lo < 0 ? 0u : (lo > 4.0e9 ? 4000000000u : (uint32_t)lo);
  *kmax = hi > 4.0e9 ? 4000000000u : (uint32_t)hi;
}

struct KeyParams {
  const SegPair *sp;
  int nsp;
  unsigned long long ntp;
  const Tile *tiles;
  double inv_bin;
  uint32_t nhist, nbuckets, nkeys;  // key = t * nbuckets + bucket; nkeys - 1 = the wide key
};

__device__ __forceinline__ uint32_t pair_key(const KeyParams &p, unsigned long long w, TilePair *tp) {
  int s;
  uint32_t I, J;
  xns_decode_tile(p.sp, p.nsp, w, &s, &I, &J);
  const SegPair g = p.sp[s];
  tp->I = g.a0 + I;
  tp->J = g.b0 + J;
  tile_pair_range(p.tiles[tp->I], p.tiles[tp->J], p.inv_bin, &tp->kmin, &tp->kmax);
  if (tp->kmax - tp->kmin + BUCKET >= WIN) return p.nkeys - 1;
  return g.cls * p.nbuckets + min(tp->kmin, p.nhist) / BUCKET;
}

__global__ void pair_key_kernel(KeyParams p, uint32_t *__restrict__ kcnt) {
  for (unsigned long long w = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; w < p.ntp;
       w += (unsigned long long)gridDim.x * blockDim.x) {
    TilePair tp;
    atomicAdd(kcnt + pair_key(p, w, &tp), 1u);
  }
}

__global__ void pair_scatter_kernel(KeyParams p, const uint32_t *__restrict__ koff, uint32_t *__restrict__ kcur,
                                    TilePair *__restrict__ list) {
  for (unsigned long long w = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; w < p.ntp;
       w += (unsigned long long)gridDim.x * blockDim.x) {
    TilePair tp;
    const uint32_t key = pair_key(p, w, &tp);
    list[koff[key] + atomicAdd(kcur + key, 1u)] = tp;
  }
}

struct HistParams {
  const double *X, *Y, *Z;  // cell-sorted coordinates
  const Tile *tiles;
  const TilePair *list;
  const CtaRange *ranges;
  unsigned long long *hist;
  unsigned int *n_bad;
  double bin, inv_bin, margin;
  uint32_t nhist, nel;
  uint32_t wide_begin, wide_end;
};

// One warp counts the pairs of one tile pair: the I tile is staged in the warp's shared memory, the J
// tile sits in registers (atoms lane and lane + 32), the warp walks i.
template <bool SAME, class Count>
__device__ __forceinline__ unsigned count_tile_pair_t(const HistParams &p, const TilePair tp, double *wI, Count count) {
  const uint32_t lane = threadIdx.x & 31;
  const Tile TI = p.tiles[tp.I], TJ = p.tiles[tp.J];
  const uint32_t ni = TI.count, nj = TJ.count;
  for (uint32_t i = lane; i < ni; i += 32) {
    wI[i] = p.X[TI.start + i];
    wI[TILE_MAX + i] = p.Y[TI.start + i];
    wI[2 * TILE_MAX + i] = p.Z[TI.start + i];
  }
  const uint32_t j0 = lane, j1 = lane + 32;
  const double x0 = j0 < nj ? p.X[TJ.start + j0] : 0.0, y0 = j0 < nj ? p.Y[TJ.start + j0] : 0.0,
               z0 = j0 < nj ? p.Z[TJ.start + j0] : 0.0;
  const double x1 = j1 < nj ? p.X[TJ.start + j1] : 0.0, y1 = j1 < nj ? p.Y[TJ.start + j1] : 0.0,
               z1 = j1 < nj ? p.Z[TJ.start + j1] : 0.0;
  __syncwarp();
  const double nh1 = (double)p.nhist - 1.0;
  unsigned bad = 0;
  // rows i and i+1 against columns j0 and j1: four independent FP64 chains per iteration, no branch
  // until the rare exact fallback.  SAME (a tile against itself) keeps only i < j.
  const bool c0 = j0 < nj, c1 = j1 < nj;
  for (uint32_t i = 0; i < ni; i += 2) {
    const uint32_t i1 = min(i + 1, ni - 1);
    const double xa = wI[i], ya = wI[TILE_MAX + i], za = wI[2 * TILE_MAX + i];
    const double xb = wI[i1], yb = wI[TILE_MAX + i1], zb = wI[2 * TILE_MAX + i1];
    const bool r1 = i + 1 < ni;
    bool v0 = c0, v1 = c1, v2 = c0 && r1, v3 = c1 && r1;
    if (SAME) {
      v0 = v0 && i < j0;
      v1 = v1 && i < j1;
      v2 = v2 && i + 1 < j0;
      v3 = v3 && i + 1 < j1;
    }
    const double d0 = ref_dist2(xa, ya, za, x0, y0, z0), d1 = ref_dist2(xa, ya, za, x1, y1, z1);
    const double d2 = ref_dist2(xb, yb, zb, x0, y0, z0), d3 = ref_dist2(xb, yb, zb, x1, y1, z1);
    uint32_t k0, k1, k2, k3;
    const bool f0 = ref_bin_fast(d0, p.inv_bin, p.margin, nh1, &k0), f1 = ref_bin_fast(d1, p.inv_bin, p.margin, nh1, &k1);
    const bool f2 = ref_bin_fast(d2, p.inv_bin, p.margin, nh1, &k2), f3 = ref_bin_fast(d3, p.inv_bin, p.margin, nh1, &k3);
    if (!((f0 || !v0) && (f1 || !v1) && (f2 || !v2) && (f3 || !v3))) {
      // a distance within the margin of a bin edge (or outside the estimate's range): exact path;
      // a bin beyond the histogram is reported, not counted
      if (v0 && !f0) { k0 = ref_bin(d0, p.bin, p.inv_bin, p.margin, p.nhist); if (k0 >= p.nhist) { v0 = false; bad++; } }
      if (v1 && !f1) { k1 = ref_bin(d1, p.bin, p.inv_bin, p.margin, p.nhist); if (k1 >= p.nhist) { v1 = false; bad++; } }
      if (v2 && !f2) { k2 = ref_bin(d2, p.bin, p.inv_bin, p.margin, p.nhist); if (k2 >= p.nhist) { v2 = false; bad++; } }
      if (v3 && !f3) { k3 = ref_bin(d3, p.bin, p.inv_bin, p.margin, p.nhist); if (k3 >= p.nhist) { v3 = false; bad++; } }
    }
    if (v0) count(k0);
    if (v1) count(k1);
    if (v2) count(k2);
    if (v3) count(k3);
  }
  __syncwarp();
  return bad;
}

template <class Count>
__device__ __forceinline__ unsigned count_tile_pair(const HistParams &p, const TilePair tp, double *wI, Count count) {
  return tp.I == tp.J ? count_tile_pair_t<true>(p, tp, wI, count) : count_tile_pair_t<false>(p, tp, wI, count);
}

// Slot s of the window holds bin B + s.  flush_window adds slots [lo, hi) (bins B + lo ...) to the
// global histogram and clears them (all threads of the CTA).
__device__ __forceinline__ void flush_window(uint32_t *win, unsigned long long *h, uint32_t B, uint32_t lo, uint32_t hi,
                                             uint32_t nhist) {
  hi = min(hi, nhist > B ? nhist - B : 0u);
  for (uint32_t s = lo + threadIdx.x; s < hi; s += HW_THREADS) {
    const uint32_t v = win[s];
    if (v) {
      atomicAdd(h + B + s, (unsigned long long)v);
      win[s] = 0;
    }
  }
}

// Moves the window from B to nb > B: bins [B, nb) leave (flushed), bins [nb, B + WIN) move down to
// slots [0, B + WIN - nb), the vacated top slots are cleared.  Called by all threads between barriers.
__device__ __forceinline__ void slide_window(uint32_t *win, unsigned long long *h, uint32_t B, uint32_t nb, uint32_t nhist) {
  const uint32_t delta = nb - B;
  flush_window(win, h, B, 0, min(delta, WIN), nhist);
  if (delta >= WIN) return;  // everything left; the flush cleared it
  __syncthreads();
  // shift down by delta in chunks: a chunk's reads lie above every slot written so far
  for (uint32_t c = 0; c < WIN - delta; c += HW_THREADS) {
    const uint32_t s = c + threadIdx.x;
    const uint32_t v = s < WIN - delta ? win[s + delta] : 0u;
    __syncthreads();
    if (s < WIN - delta) win[s] = v;
    __syncthreads();
  }
  for (uint32_t s = WIN - delta + threadIdx.x; s < WIN; s += HW_THREADS) win[s] = 0;
}

__global__ void __launch_bounds__(HW_THREADS, 1) hist_window_kernel(HistParams p) {
  extern __shared__ uint32_t win[];  // WIN bins, then HW_WARPS staging areas of 3 x 64 doubles
  double *wI = reinterpret_cast<double *>(win + WIN) + (threadIdx.x >> 5) * 3 * TILE_MAX;
  const CtaRange rg = p.ranges[blockIdx.x];
  if (rg.begin >= rg.end) return;
  unsigned long long *h = p.hist + (size_t)rg.type * p.nhist;
  for (uint32_t s = threadIdx.x; s < WIN; s += HW_THREADS) win[s] = 0;
  uint32_t B = p.list[rg.begin].kmin / BUCKET * BUCKET;
  __syncthreads();
  unsigned bad = 0;
  for (uint32_t r = rg.begin; r < rg.end; r += HW_WARPS) {
    // the round's entries must fit the window [B, B + WIN): slide it when the farthest one does not
    uint32_t kmax = 0;
    for (uint32_t e = r; e < min(r + HW_WARPS, rg.end); e++) kmax = max(kmax, p.list[e].kmax);
    if (kmax >= B + WIN) {
      const uint32_t nb = p.list[r].kmin / BUCKET * BUCKET;
      if (nb > B) {
        __syncthreads();
        slide_window(win, h, B, nb, p.nhist);
        B = nb;
        __syncthreads();
      }
    }
    const uint32_t e = r + (threadIdx.x >> 5);
    if (e < rg.end) {
      const uint32_t base = B;
      bad += count_tile_pair(p, p.list[e], wI, [&](uint32_t k) {
        const uint32_t s = k - base;
        if (s < WIN) atomicAdd(win + s, 1u);
        else atomicAdd(h + k, 1ull);  // outside the window (a round spanning two buckets): count directly
      });
    }
  }
  __syncthreads();
  flush_window(win, h, B, 0, WIN, p.nhist);
  if (bad) atomicAdd(p.n_bad, bad);
}

__global__ void __launch_bounds__(256) hist_wide_kernel(HistParams p) {
  __shared__ double stage[8 * 3 * TILE_MAX];
  double *wI = stage + (threadIdx.x >> 5) * 3 * TILE_MAX;
  unsigned bad = 0;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t e = p.wide_begin + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); e < p.wide_end; e += nw) {
    const TilePair tp = p.list[e];
    const uint32_t a = min(p.tiles[tp.I].elem, p.tiles[tp.J].elem), b = max(p.tiles[tp.I].elem, p.tiles[tp.J].elem);
    unsigned long long *h = p.hist + (size_t)(a * p.nel - a * (a - 1) / 2 + (b - a)) * p.nhist;
    bad += count_tile_pair(p, tp, wI, [&](uint32_t k) { atomicAdd(h + k, 1ull); });
  }
  if (bad) atomicAdd(p.n_bad, bad);
}

}  // namespace

int xns_hist_device(xns_ctx *ctx, const DevCoords &dc, uint32_t nhist, double bin, unsigned long long *d_hist) {
  const uint32_t nel = (uint32_t)dc.n_el.size();
  if (nhist == 0 || !(bin > 0)) return xns_fail(ctx, XNS_ERR_ARG, "histogram: nhist == 0 or bin <= 0");
  const uint32_t P = xns_npairs(nel);
  int st;
  XNS_CUDA(ctx, cudaMemsetAsync(d_hist, 0, sizeof(unsigned long long) * (size_t)P * nhist, ctx->stream));
  void *flags;
  if ((st = xns_scratch(ctx, SLOT_FLAGS, 64, &flags))) return st;
  XNS_CUDA(ctx, cudaMemsetAsync(flags, 0, 64, ctx->stream));
  if (dc.ntot < 2) return XNS_OK;

  // -- element bounding boxes -> cell grids
  void *vkey, *vh;
  const size_t small_bytes = sizeof(ElemGrid) * nel + 2 * 3 * sizeof(unsigned long long) * nel + 64;
  if ((st = xns_scratch(ctx, SLOT_AUX, small_bytes, &vkey))) return st;
  ElemGrid *d_eg = (ElemGrid *)vkey;
  unsigned long long *d_bmin = (unsigned long long *)(d_eg + nel), *d_bmax = d_bmin + 3 * nel;
  if ((st = xns_pinned(ctx, small_bytes, &vh))) return st;
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  std::vector<ElemGrid> eg(nel);
  for (uint32_t e = 0; e < nel; e++) {
    memset(&eg[e], 0, sizeof(ElemGrid));
    eg[e].atom0 = dc.off_el[e];
    eg[e].natoms = dc.n_el[e];
  }
  memcpy(vh, eg.data(), sizeof(ElemGrid) * nel);
  XNS_CUDA(ctx, cudaMemcpyAsync(d_eg, vh, sizeof(ElemGrid) * nel, cudaMemcpyHostToDevice, ctx->stream));
  XNS_CUDA(ctx, cudaMemsetAsync(d_bmin, 0xff, 3 * sizeof(unsigned long long) * nel, ctx->stream));
  XNS_CUDA(ctx, cudaMemsetAsync(d_bmax, 0, 3 * sizeof(unsigned long long) * nel, ctx->stream));
  elem_bbox_kernel<<<dim3(std::max(1, ctx->num_sms / (int)nel), nel), 256, 0, ctx->stream>>>(dc.x, dc.y, dc.z, d_eg, d_bmin,
                                                                                             d_bmax);
  XNS_LAUNCHED(ctx);
  std::vector<unsigned long long> bb(6 * nel);
  XNS_CUDA(ctx, cudaMemcpyAsync(bb.data(), d_bmin, 6 * sizeof(unsigned long long) * nel, cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  uint32_t ncells = 0;
  for (uint32_t e = 0; e < nel; e++) {
    ElemGrid &g = eg[e];
    g.base = ncells;
    if (!g.natoms) continue;
    double ext[3], vol = 1;
    for (int k = 0; k < 3; k++) {
      g.o[k] = ord_value(bb[3 * e + k]);
      ext[k] = ord_value(bb[3 * nel + 3 * e + k]) - g.o[k];
      if (!(ext[k] >= 0) || !std::isfinite(ext[k])) return xns_fail(ctx, XNS_ERR_ARG, "histogram: non-finite coordinates");
    }
    const double emax = std::max(ext[0], std::max(ext[1], ext[2]));
    for (int k = 0; k < 3; k++) vol *= std::max(ext[k], 1e-3 * emax + 1e-9);
    const double s = std::max(cbrt(CELL_TARGET * vol / g.natoms), 1e-6);
    for (int k = 0; k < 3; k++) {
      g.n[k] = (uint32_t)std::min<double>(MAX_CELLS_AXIS, std::max(1.0, floor(ext[k] / s) + 1));
      g.inv[k] = ext[k] > 0 ? g.n[k] / (ext[k] * (1 + 1e-12)) : 0.0;
    }
    ncells += g.n[0] * g.n[1] * g.n[2];
  }

  // -- counting sort of atoms by cell
  void *vcell, *vsort;
  if ((st = xns_scratch(ctx, SLOT_HCELL, sizeof(uint32_t) * (4 * (size_t)ncells + 8), &vcell))) return st;
  uint32_t *d_cnt = (uint32_t *)vcell, *d_coff = d_cnt + ncells, *d_toff = d_coff + ncells, *d_cur = d_toff + ncells,
           *d_tot = d_cur + ncells;
  if ((st = xns_scratch(ctx, SLOT_HSORT, (sizeof(double) * 3 + sizeof(uint32_t)) * (size_t)dc.ntot, &vsort))) return st;
  double *Xs = (double *)vsort, *Ys = Xs + dc.ntot, *Zs = Ys + dc.ntot;
  uint32_t *d_cid = (uint32_t *)(Zs + dc.ntot);
  memcpy(vh, eg.data(), sizeof(ElemGrid) * nel);
  XNS_CUDA(ctx, cudaMemcpyAsync(d_eg, vh, sizeof(ElemGrid) * nel, cudaMemcpyHostToDevice, ctx->stream));
  XNS_CUDA(ctx, cudaMemsetAsync(d_cnt, 0, sizeof(uint32_t) * ncells, ctx->stream));
  XNS_CUDA(ctx, cudaMemsetAsync(d_cur, 0, sizeof(uint32_t) * ncells, ctx->stream));
  const int gx = std::max(1, ctx->num_sms * 4 / (int)nel);
  cell_count_kernel<<<dim3(gx, nel), 256, 0, ctx->stream>>>(dc.x, dc.y, dc.z, d_eg, d_cid, d_cnt);
  XNS_LAUNCHED(ctx);
  scan_kernel<<<1, SCAN_THREADS, 0, ctx->stream>>>(d_cnt, ncells, d_coff, d_toff, d_tot);
  XNS_LAUNCHED(ctx);
  cell_scatter_kernel<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(dc.x, dc.y, dc.z, dc.ntot, d_cid, d_coff, d_cur, Xs, Ys, Zs);
  XNS_LAUNCHED(ctx);
  // tiles per element: read the tile offsets at the element boundaries
  std::vector<uint32_t> tstart(nel + 1);
  uint32_t totals[2];
  XNS_CUDA(ctx, cudaMemcpyAsync(totals, d_tot, sizeof(totals), cudaMemcpyDeviceToHost, ctx->stream));
  for (uint32_t e = 0; e < nel; e++)
    if (eg[e].base < ncells)
      XNS_CUDA(ctx, cudaMemcpyAsync(&tstart[e], d_toff + eg[e].base, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const uint32_t ntiles = totals[1];
  for (uint32_t e = 0; e < nel; e++)
    if (eg[e].base >= ncells) tstart[e] = ntiles;
  tstart[nel] = ntiles;
  void *vtile;
  if ((st = xns_scratch(ctx, SLOT_HTILE, sizeof(Tile) * (size_t)std::max(ntiles, 1u), &vtile))) return st;
  Tile *d_tiles = (Tile *)vtile;
  tile_build_kernel<<<(ncells + 255) / 256, 256, 0, ctx->stream>>>(d_cnt, d_coff, d_toff, ncells, d_eg, nel, d_tiles);
  XNS_LAUNCHED(ctx);
  tile_bbox_kernel<<<(ntiles + 7) / 8, 256, 0, ctx->stream>>>(Xs, Ys, Zs, d_tiles, ntiles);
  XNS_LAUNCHED(ctx);

  // -- tile pairs sorted by (element pair, distance bucket)
  std::vector<Segment> sa, sb;
  std::vector<uint32_t> cls, same;
  uint32_t t = 0;
  for (uint32_t a = 0; a < nel; a++)
    for (uint32_t b = a; b < nel; b++, t++) {
      sa.push_back({tstart[a], tstart[a + 1] - tstart[a]});
      sb.push_back({tstart[b], tstart[b + 1] - tstart[b]});
      cls.push_back(t);
      same.push_back(a == b);
    }
  std::vector<SegPair> sched;
  const unsigned long long ntp = xns_build_schedule(sa, sb, cls, same, 1, 1, &sched);
  if (ntp >= (1ull << 32)) return xns_fail(ctx, XNS_ERR_ARG, "histogram: too many tile pairs");
  if (ntp == 0) return XNS_OK;
  SegPair *d_sp;
  if ((st = xns_upload_schedule(ctx, sched, &d_sp))) return st;
  KeyParams kp;
  kp.sp = d_sp;
  kp.nsp = (int)sched.size();
  kp.ntp = ntp;
  kp.tiles = d_tiles;
  kp.inv_bin = 1.0 / bin;
  kp.nhist = nhist;
  kp.nbuckets = nhist / BUCKET + 1;
  kp.nkeys = P * kp.nbuckets + 1;
  void *vk, *vl;
  if ((st = xns_scratch(ctx, SLOT_HKEY, sizeof(uint32_t) * (3 * (size_t)kp.nkeys + 8), &vk))) return st;
  uint32_t *d_kcnt = (uint32_t *)vk, *d_koff = d_kcnt + kp.nkeys, *d_kcur = d_koff + kp.nkeys, *d_ktot = d_kcur + kp.nkeys;
  if ((st = xns_scratch(ctx, SLOT_HLIST, sizeof(TilePair) * ntp, &vl))) return st;
  TilePair *d_list = (TilePair *)vl;
  XNS_CUDA(ctx, cudaMemsetAsync(d_kcnt, 0, sizeof(uint32_t) * kp.nkeys, ctx->stream));
  XNS_CUDA(ctx, cudaMemsetAsync(d_kcur, 0, sizeof(uint32_t) * kp.nkeys, ctx->stream));
  const int kgrid = ctx->num_sms * 8;
  pair_key_kernel<<<kgrid, 256, 0, ctx->stream>>>(kp, d_kcnt);
  XNS_LAUNCHED(ctx);
  scan_kernel<<<1, SCAN_THREADS, 0, ctx->stream>>>(d_kcnt, kp.nkeys, d_koff, nullptr, d_ktot);
  XNS_LAUNCHED(ctx);
  pair_scatter_kernel<<<kgrid, 256, 0, ctx->stream>>>(kp, d_koff, d_kcur, d_list);
  XNS_LAUNCHED(ctx);
  // split the sorted list into CTA ranges, one element pair per CTA, in proportion to its pairs
  std::vector<uint32_t> koff(kp.nkeys);
  XNS_CUDA(ctx, cudaMemcpyAsync(koff.data(), d_koff, sizeof(uint32_t) * kp.nkeys, cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const uint32_t n_narrow = koff[kp.nkeys - 1];
  // a CTA's u32 window counts at most 64*64*entries pairs per bin: keep that below 2^31
  const uint32_t max_per_cta = (1u << 19);
  const int G = std::max<int>(ctx->num_sms, (int)((n_narrow + max_per_cta - 1) / max_per_cta));
  // CTAs per element pair in proportion to its entries (largest remainders get the spare CTAs), so
  // that one wave of G CTAs covers the list
  std::vector<uint32_t> nty(P), gty(P, 0);
  int used = 0;
  for (uint32_t ty = 0; ty < P; ty++) {
    nty[ty] = koff[(ty + 1) * kp.nbuckets] - koff[ty * kp.nbuckets];
    if (nty[ty]) {
      gty[ty] = std::max(1u, (uint32_t)((double)G * nty[ty] / std::max(n_narrow, 1u)));
      used += gty[ty];
    }
  }
  while (used < G) {
    uint32_t best = 0;
    double most = -1;
    for (uint32_t ty = 0; ty < P; ty++)
      if (nty[ty] && (double)nty[ty] / gty[ty] > most) {
        most = (double)nty[ty] / gty[ty];
        best = ty;
      }
    if (most < 0) break;
    gty[best]++;
    used++;
  }
  std::vector<CtaRange> ranges;
  for (uint32_t ty = 0; ty < P; ty++) {
    if (!nty[ty]) continue;
    const uint32_t b0 = koff[ty * kp.nbuckets], b1 = b0 + nty[ty];
    const uint32_t L = (nty[ty] + gty[ty] - 1) / gty[ty];
    for (uint32_t s = b0; s < b1; s += L) ranges.push_back({s, std::min(b1, s + L), ty, 0});
  }
  HistParams hp;
  hp.X = Xs;
  hp.Y = Ys;
  hp.Z = Zs;
  hp.tiles = d_tiles;
  hp.list = d_list;
  hp.hist = d_hist;
  hp.n_bad = (unsigned int *)flags;
  hp.bin = bin;
  hp.inv_bin = 1.0 / bin;
  hp.margin = (double)nhist * ldexp(1.0, -37);
  hp.nhist = nhist;
  hp.nel = nel;
  hp.wide_begin = n_narrow;
  hp.wide_end = (uint32_t)ntp;
  if (!ranges.empty()) {
    void *vr, *vrh;
    if ((st = xns_scratch(ctx, SLOT_SEGPAIRS, sizeof(CtaRange) * ranges.size() + sizeof(SegPair) * sched.size(), &vr)))
      return st;
    // the schedule is no longer needed once the list is built; its slot now holds the CTA ranges
    if ((st = xns_pinned(ctx, sizeof(CtaRange) * ranges.size(), &vrh))) return st;
    XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    memcpy(vrh, ranges.data(), sizeof(CtaRange) * ranges.size());
    XNS_CUDA(ctx, cudaMemcpyAsync(vr, vrh, sizeof(CtaRange) * ranges.size(), cudaMemcpyHostToDevice, ctx->stream));
    hp.ranges = (const CtaRange *)vr;
    const size_t smem = sizeof(uint32_t) * WIN + sizeof(double) * 3 * TILE_MAX * HW_WARPS;
    XNS_CUDA(ctx, cudaFuncSetAttribute(hist_window_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if ((st = xns_stage_begin(ctx, STAGE_HIST))) return st;
    hist_window_kernel<<<(unsigned)ranges.size(), HW_THREADS, smem, ctx->stream>>>(hp);
    XNS_LAUNCHED(ctx);
  }
  if (ranges.empty() && (st = xns_stage_begin(ctx, STAGE_HIST))) return st;
  if (hp.wide_end > hp.wide_begin) {
    hist_wide_kernel<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(hp);
    XNS_LAUNCHED(ctx);
  }
  if ((st = xns_stage_end(ctx, STAGE_HIST))) return st;
  unsigned int bad = 0;
  XNS_CUDA(ctx, cudaMemcpyAsync(&bad, flags, sizeof(bad), cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (bad) return xns_fail(ctx, XNS_ERR_RANGE, "histogram: " + std::to_string(bad) + " pair distances fall beyond nhist bins");
  return XNS_OK;
}

extern "C" int xns_calc_hist(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel, uint32_t nhist,
                             double bin, uint64_t *hist) {
  if (!ctx) return XNS_ERR_ARG;
  if (!hist) return xns_fail(ctx, XNS_ERR_ARG, "hist: null output");
  int st;
  DevCoords dc;
  if ((st = xns_upload_coords(ctx, xyz_el, n_el, nel, &dc))) return st;
  void *d_hist;
  size_t bytes = sizeof(unsigned long long) * (size_t)xns_npairs(nel) * nhist;
  if ((st = xns_scratch(ctx, SLOT_HIST, bytes, &d_hist))) return st;
  if ((st = xns_timer_start(ctx))) return st;
  if ((st = xns_hist_device(ctx, dc, nhist, bin, (unsigned long long *)d_hist))) return st;
  if ((st = xns_timer_stop(ctx))) return st;
  XNS_CUDA(ctx, cudaMemcpyAsync(hist, d_hist, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XNS_OK;
}
