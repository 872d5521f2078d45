// Pair-distance histogram (replaces calcHist, CalcFunctions.cpp:757-809, and calcHistKernel,
// CalcFunctionsCUDA.cu:814-920), for one structure or a set of independent structures at once.
//
// Counts are bit-identical to the reference's.  At the reference's 0.001 A bins a 2e5-atom structure
// has ~3e5 bins per element pair: far more than a shared-memory histogram holds, and one global atomic
// per pair leaves the kernel bound by L2 atomics.  So the pairs are ordered by distance first:
//   1. atoms of each element are counting-sorted into cells of ~cell_target atoms, on the one of six
//      candidate grids whose tiles waste the fewest warp lanes (cand_count / cand_slots, then
//      cell_count / scan / cell_scatter); each cell is cut into tiles of <= 64 atoms with a bounding
//      box (tile_build / tile_bbox);
//   2. every tile pair (upper triangle within an element, all pairs across elements of the same
//      structure) gets the bin range [kmin, kmax] its bounding boxes allow, and is counting-sorted by
//      (class, kmin / BUCKET), a class being one element pair of one structure (pair_key / scan /
//      pair_scatter);
//   3. the sorted list is cut into runs of one class; hist_window_kernel is persistent (one CTA per
//      SM) and takes runs from a work queue, largest first, one tile pair per warp, counting into a
//      window of u32 bins in shared memory that slides up the distance axis (bins that leave the
//      window are added to the u64 global histogram once per run);
//   4. hist_wide_kernel: tile pairs whose range is wider than the window (sparse elements) count
//      straight into the global histogram.
//
// Bin decision, per pair: an FP32 estimate of r/bin with a proven error bound (count_tile_pair_t: a
// centred estimate for tile pairs far apart, whose error scales with the tile size; a direct one
// otherwise), computed for two pairs at a time on packed f32x2 pairs.  Pairs whose estimate lies
// within the bound of a bin edge (about 0.75 % of the benchmark's), near the last bin or outside the
// window are queued per warp and binned exactly, 32 at a time, with FP64 in the reference's operation
// order (hist_bin.cuh).  Atom order inside a cell and list order inside a bucket come from atomics,
// but counts do not depend on either.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cmath>

#include "hist_bin.cuh"
#include "f32x2.cuh"
#include "hist_set.cuh"
#include "schedule.cuh"

using namespace xns_hist;

namespace {

constexpr int TILE_MAX = 64;         // atoms per tile
constexpr int MAX_CELLS_AXIS = 256;
constexpr int HW_WARPS = 20;         // at 96 registers a thread, 20 warps fill the register file
constexpr int HW_THREADS = 32 * HW_WARPS;
constexpr uint32_t WIN_MAX = HIST_WIN_MAX;  // largest window (bins) that fits with the warp stages
constexpr uint32_t BUCKET = 1024;    // distance bucket of the tile-pair sort, in bins
constexpr int SCAN_THREADS = 1024;
constexpr int QUEUE = 64;            // queue entries per warp: u32 (i/4) << 13 | lane << 8 | 8-bit pair mask
// per warp: FP64 I tile, FP32 I-tile offsets (+ P_i), the queue (bytes)
constexpr int WARP_STAGE = 3 * TILE_MAX * 8 + 4 * TILE_MAX * 4 + QUEUE * 4;
// the window kernel's shared memory (window, 32 spare slots, stages, 16 static bytes) within 227 KB
static_assert(4 * (WIN_MAX + 32) + WARP_STAGE * HW_WARPS + 16 <= 227 * 1024, "window and stages fit");

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
// Class of an element's pairs: structure's first class, element index within the structure, the
// structure's element count.
struct ElemCls {
  uint32_t cls_base, local, nel_s, pad;
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
      // fmin / fmax skip a NaN: it widens the box to infinity instead, so that the plan rejects it
      const bool nan = !(v[k] == v[k]);
      mn[k] = fmin(mn[k], nan ? -INFINITY : v[k]);
      mx[k] = fmax(mx[k], nan ? INFINITY : v[k]);
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
                                    double *__restrict__ Zs, uint32_t *__restrict__ idx) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t c = cid[i];
    const uint32_t p = cell_off[c] + atomicAdd(cursor + c, 1u);
    Xs[p] = X[i];
    Ys[p] = Y[i];
    Zs[p] = Z[i];
    if (idx) idx[p] = i;
  }
}

// The scatter's order inside a cell depends on the atomics; a sharded plan needs the same tiles in every
// shard, so it puts each cell's atoms back in input order (one thread per cell, insertion sort).
__global__ void cell_order_kernel(uint32_t ncells, const uint32_t *__restrict__ cell_off, const uint32_t *__restrict__ cnt,
                                  double *__restrict__ Xs, double *__restrict__ Ys, double *__restrict__ Zs,
                                  uint32_t *__restrict__ idx) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  const uint32_t b = cell_off[c], e = b + cnt[c];
  for (uint32_t m = b + 1; m < e; m++) {
    const uint32_t k = idx[m];
    const double x = Xs[m], y = Ys[m], z = Zs[m];
    uint32_t t = m;
    for (; t > b && idx[t - 1] > k; t--) idx[t] = idx[t - 1], Xs[t] = Xs[t - 1], Ys[t] = Ys[t - 1], Zs[t] = Zs[t - 1];
    idx[t] = k, Xs[t] = x, Ys[t] = y, Zs[t] = z;
  }
}

// dst[i] = src[idx[i]]
__global__ void gather_u32_kernel(const uint32_t *__restrict__ src, const uint32_t *__restrict__ idx, uint32_t n,
                                  uint32_t *__restrict__ dst) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[idx[i]];
}

// Candidate cell grids (NCAND per element, cg[e * NCAND + c], cells counted from cg[].base): atoms per
// cell, then the warp lanes that the grid's tiles would occupy, 64 per tile (the counting kernel walks
// a J tile with 64 lanes whatever its size).
constexpr int NCAND = 6;
__global__ void cand_count_kernel(const double *__restrict__ X, const double *__restrict__ Y, const double *__restrict__ Z,
                                  const ElemGrid *__restrict__ cg, uint32_t *__restrict__ cnt) {
  const ElemGrid g = cg[blockIdx.y * NCAND + blockIdx.z];
  for (uint32_t i = g.atom0 + blockIdx.x * blockDim.x + threadIdx.x; i < g.atom0 + g.natoms; i += gridDim.x * blockDim.x)
    atomicAdd(cnt + cell_of(g, X[i], Y[i], Z[i]), 1u);
}
__global__ void cand_slots_kernel(const uint32_t *__restrict__ cnt, const ElemGrid *__restrict__ cg,
                                  unsigned long long *__restrict__ slots) {
  const ElemGrid g = cg[blockIdx.x];
  const uint32_t nc = g.n[0] * g.n[1] * g.n[2];
  unsigned long long t = 0;
  for (uint32_t c = threadIdx.x; c < nc; c += blockDim.x) t += (cnt[g.base + c] + TILE_MAX - 1) / TILE_MAX;
  for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if ((threadIdx.x & 31) == 0 && t) atomicAdd(slots + blockIdx.x, t * TILE_MAX);
}

// Cells -> tiles: a cell of n atoms becomes ceil(n/64) tiles of near-equal size.
__global__ void tile_build_kernel(const uint32_t *__restrict__ cnt, const uint32_t *__restrict__ cell_off,
                                  const uint32_t *__restrict__ tile_off, uint32_t ncells, const ElemGrid *__restrict__ eg,
                                  uint32_t nel, Tile *__restrict__ tiles) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells; c += gridDim.x * blockDim.x) {
    const uint32_t n = cnt[c];
    if (!n) continue;
    uint32_t lo = 0, hi = nel - 1;  // last element whose first cell is <= c
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (eg[mid].base <= c) lo = mid;
      else hi = mid - 1;
    }
    const uint32_t nt = (n + TILE_MAX - 1) / TILE_MAX;
    uint32_t s = cell_off[c];
    for (uint32_t t = 0; t < nt; t++) {
      const uint32_t cnt_t = n / nt + (t < n % nt ? 1 : 0);
      Tile tl;
      tl.start = s;
      tl.count = cnt_t;
      tl.elem = lo;
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
  unsigned long long ntp;   // tile pairs of this pass: w = wbeg + [0, ntp)
  unsigned long long wbeg;
  const Tile *tiles;
  double inv_bin;
  uint32_t nhist, nbuckets, nkeys;  // key = class * nbuckets + bucket; nkeys - 1 = the wide key
  uint32_t win;                     // window bins of the counting kernel
  uint32_t shard, nshard;           // this plan keeps the tile pairs w with w % nshard == shard
};

__device__ __forceinline__ uint32_t pair_key(const KeyParams &p, unsigned long long w, TilePair *tp) {
  int s;
  uint32_t I, J;
  xns_decode_tile(p.sp, p.nsp, w, &s, &I, &J);
  const SegPair g = p.sp[s];
  tp->I = g.a0 + I;
  tp->J = g.b0 + J;
  tile_pair_range(p.tiles[tp->I], p.tiles[tp->J], p.inv_bin, &tp->kmin, &tp->kmax);
  if (tp->kmax - tp->kmin + BUCKET >= p.win) return p.nkeys - 1;
  return g.cls * p.nbuckets + min(tp->kmin, p.nhist) / BUCKET;
}

// Consecutive tile pairs (a tile against its neighbours' tiles) mostly share a distance bucket, so the
// lanes of a warp group by key (match.any) and one lane per key does the warp's atomic.
// The key pass decodes every tile pair once, counts its key and keeps the tile pair and key (tmp, tkey:
// indexed by the pass-local w; key ~0u for a tile pair of another shard); the scatter pass only moves them.
__global__ void pair_key_kernel(KeyParams p, uint32_t *__restrict__ kcnt, TilePair *__restrict__ tmp,
                                uint32_t *__restrict__ tkey) {
  const uint32_t lane = threadIdx.x & 31;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long w0 = blockIdx.x * (unsigned long long)blockDim.x + (threadIdx.x & ~31u); w0 < p.ntp;
       w0 += stride) {
    const unsigned long long wl = w0 + lane, w = p.wbeg + wl;
    const bool act = wl < p.ntp && (p.nshard == 1 || w % p.nshard == p.shard);
    const unsigned act_mask = __ballot_sync(0xffffffffu, act);
    if (act) {
      TilePair tp;
      const uint32_t key = pair_key(p, w, &tp);
      const unsigned same = __match_any_sync(act_mask, key);
      if (lane == (uint32_t)(__ffs(same) - 1)) atomicAdd(kcnt + key, (uint32_t)__popc(same));
      tmp[wl] = tp;
      tkey[wl] = key;
    } else if (wl < p.ntp) {
      tkey[wl] = 0xffffffffu;
    }
  }
}

__global__ void pair_scatter_kernel(KeyParams p, const uint32_t *__restrict__ koff, uint32_t *__restrict__ kcur,
                                    const TilePair *__restrict__ tmp, const uint32_t *__restrict__ tkey,
                                    TilePair *__restrict__ list) {
  const uint32_t lane = threadIdx.x & 31;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long w0 = blockIdx.x * (unsigned long long)blockDim.x + (threadIdx.x & ~31u); w0 < p.ntp;
       w0 += stride) {
    const unsigned long long wl = w0 + lane;
    const uint32_t key = wl < p.ntp ? tkey[wl] : 0xffffffffu;
    const bool act = key != 0xffffffffu;
    const unsigned act_mask = __ballot_sync(0xffffffffu, act);
    if (act) {
      const unsigned same = __match_any_sync(act_mask, key);
      const uint32_t leader = (uint32_t)(__ffs(same) - 1);
      uint32_t at = 0;
      if (lane == leader) at = atomicAdd(kcur + key, (uint32_t)__popc(same));
      at = __shfl_sync(same, at, leader) + (uint32_t)__popc(same & ((1u << lane) - 1u));
      list[koff[key] + at] = tmp[wl];
    }
  }
}

struct HistParams {
  const double *X, *Y, *Z;  // cell-sorted coordinates
  const Tile *tiles;
  const TilePair *list;
  const CtaRange *ranges;
  const ElemCls *ecls;
  unsigned int *queue;      // next run for the persistent window kernel
  unsigned long long *hist; // classes x nhist
  unsigned int *n_bad;
  double bin, inv_bin, margin;
  uint32_t nhist, nranges;
  uint32_t wide_begin, wide_end;
  uint32_t win;             // window bins (<= WIN_MAX)
};
static_assert(sizeof(HistParams) <= sizeof(((HistLaunch *)0)->params), "HistLaunch holds the kernel parameters");

// Geometry of a tile pair in bins: centres' offset D = (c_I - c_J)/bin, R0 = |D|, per-axis half
// extents E (+1 bin against rounding) and the radii rho = |E| of the boxes around the centres.
struct PairGeom {
  double D[3], R0;
  float EI, EJ, rhoI, rhoJ;
};
__device__ __forceinline__ PairGeom pair_geom(const Tile &TI, const Tile &TJ, double ib) {
  PairGeom g;
  double r2 = 0;
  float eI2 = 0.f, eJ2 = 0.f;
  g.EI = 0.f;
  g.EJ = 0.f;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    g.D[k] = (0.5 * (TI.lo[k] + TI.hi[k]) - 0.5 * (TJ.lo[k] + TJ.hi[k])) * ib;
    // half extents rounded up by a part in 1e6 (bounds, not values)
    const float eI = (float)(0.5 * (TI.hi[k] - TI.lo[k]) * ib + 1.0) * 1.000001f;
    const float eJ = (float)(0.5 * (TJ.hi[k] - TJ.lo[k]) * ib + 1.0) * 1.000001f;
    g.EI = fmaxf(g.EI, eI);
    g.EJ = fmaxf(g.EJ, eJ);
    r2 += g.D[k] * g.D[k];
    eI2 = fmaf(eI, eI, eI2);
    eJ2 = fmaf(eJ, eJ, eJ2);
  }
  g.R0 = sqrt(r2);
  g.rhoI = sqrtf(eI2) * 1.000001f;
  g.rhoJ = sqrtf(eJ2) * 1.000001f;
  return g;
}

// Far tile pairs (R0 >= 2 (rho_I + rho_J), so every pair has r >= R0 / 2) take the centred estimate.
__device__ __forceinline__ bool far_pair(const PairGeom &g) { return g.R0 >= 2.0 * (g.rhoI + g.rhoJ); }

// One warp counts the pairs of one tile pair: the I tile's FP64 coordinates and FP32 offsets are
// staged in the warp's shared memory (stage: WARP_STAGE bytes), the J tile's sit in registers (atoms
// lane and lane + 32), the warp walks i four rows at a time (four independent chains of two packed
// pairs each).  SAME (a tile
// against itself) keeps only i < j.  Each pair gets an FP32 estimate of r/bin with a proven error
// bound; pairs whose estimate lies within the bound of a bin edge, near or beyond the last bin, or
// outside the CTA's window are appended to the warp's queue (one entry per lane and step with an
// 8-bit mask; ballot + popc: consecutive entries) and binned exactly with FP64 from the coordinates
// (hist_bin.cuh), one entry per lane, whenever 32 wait.
//
// Direct estimate (SAME and close tile pairs; u = 2^-24): dh is D rounded to float, dl its low part;
// the I offsets are (x_i - c_I)/bin and the J offsets (x_j - c_J)/bin - dl, rounded to float.  Each
// axis |dx - dx_true| <= u|dx| + C, C = u(2 E_I + 3 E_J + 2) + 2^-40 |D|; d2 by FMAs adds 3u relative;
// rsqrt.approx (2 ulp) followed by one Newton step leaves u + O(u^2) relative to sqrt(d2); so
// |r - r_true| <= 4.3 u r + 1.74 C.  With m = 6 u r + 2 C, any r whose distance d to the nearest
// integer is >= m has floor(r) equal to the reference's bin (whose own FP64 rounding is below 1e-10
// bins).  r + 1.5*2^23 rounds r to an integer in the low mantissa bits (r < 2^22), which gives
// round(r) and d without a conversion.
//
// Centred estimate (far tile pairs): with a = (x_i - c_I)/bin, b = (x_j - c_J)/bin and the bin
// midpoint R = floor(R0) + 0.5 nearest the centres' distance,
//   r^2 = R^2 + num,  num = P_i - Q_j - 2 a.b,  P_i = 2 D.a + |a|^2 + (R0^2 - R^2),  Q_j = 2 D.b - |b|^2,
// and t = r - R = r - floor(R0) - 0.5, so that floor(r) = floor(R0) + round(t).  P_i and Q_j are formed
// in FP64 per tile pair and rounded to float; per pair num = (P_i - Q_j) + a.(-2 b) in FP32,
// d2 = num + R^2, y = rsqrt(d2) and t0 = d2 y - R (one FMA: r to a few ulp, so t0 is within ~5u r of
// t), then one Newton step on t^2 + 2 R t - num = 0 whose derivative 2 r is 2 / y:
//   t = t0 + (num - t0 (t0 + 2 R)) y / 2   (a subtraction and two FMAs),
// which leaves the error of t0 only squared.  Its error (centred_margin) is K0 + K1 |t - r + R| with K0
// of order u rho and K1 about 4u: it grows with the tile size, not with r; one MUFU operation per pair.
struct CentredConsts {
  float R2, NR, N2R, K1, mc;  // R^2 rounded, -R, -2 R (both exact); fast iff |d| <= mc - K1 |t|
  int R0i;                    // floor(R0)
  double S;                   // R0^2 - R^2, added to every P_i
};
// The bound, for r >= R0 - rho_I - rho_J >= R0 / 2 (far_pair), u = 2^-24 the unit roundoff (each FP32
// rounding at most u relative), t~ = r~ - R where r~^2 = R^2 + num~ (num~ the computed num):
//   num:    |num~ - num| <= u(|P| + |Q|) + 2u|num| + 12u rho_I rho_J (P, Q and the difference rounded;
//           the dot product's roundings, |a.b| <= rho_I rho_J; the last add), with |P| <= 2 R0 rho_I +
//           rho_I^2 + R0 + 1/4 and |Q| <= 2 R0 rho_J + rho_J^2;  |t~ - t| = |num~ - num| / (r + r~), and
//           r + r~ >= 1.998 (R0 - rho_I - rho_J);  2u|num| / (r + r~) = 2u |t| (r + R) / (r + r~) <= 2uF|t|
//           with F = 1/2 + (R0 + 1/2) / (2 (R0 - rho_I - rho_J)) (at most 3/2);
//   Newton: t0 - t~ <= r (rsqrt 2.14u + d2's 5.1u / 2) + u|t0| <= 5.7u r and y within 4.7u of 1 / r~, so
//           the step leaves (t0 - t~)(4.7u + (t0 - t~) / 2r) <= 44 u^2 r;  rounding t0 + 2R costs
//           u |t0| (r + R) y / 2 <= uF|t|, the residual's rounding u^2 r more, the final FMA u|t|;
// so |t - (r - R)| <= K0 + (3F + 1) u |t - r + R| + O(u^2), K0 = the absolute part of num's bound
// divided by 1.998 (R0 - rho_I - rho_J), plus 50 u^2 (R0 + rho_I + rho_J).
// The constants are bounds: evaluated in FP32 and enlarged by 2 % (more than FP32 rounding can take away).
__device__ __forceinline__ CentredConsts centred_consts(const PairGeom &g) {
  const float u = 5.9604645e-08f;  // 2^-24
  const float R0 = (float)g.R0;
  const float rs = g.rhoI + g.rhoJ, rr = 12.0f * g.rhoI * g.rhoJ;
  const float PQ = 2.0f * R0 * rs + g.rhoI * g.rhoI + g.rhoJ * g.rhoJ + R0 + 0.25f;
  const float Lr = 1.998f * (R0 - rs) * 0.999999f;
  const float F = (0.5f + (R0 + 0.5f) / (2.0f * (R0 - rs) * 0.999999f)) * 1.000001f;
  const float K1 = (3.0f * F + 1.0f) * u * 1.02f;
  // 1e-9 for FP64 errors of D, a, P, Q and the reference's own rounding
  const float K0 = u * (PQ + rr) / Lr * 1.02f + 50.0f * u * u * (R0 + rs) * 1.02f + 1e-9f + R0 * 9.094947e-13f;
  CentredConsts c;
  const double fl = floor(g.R0), R = fl + 0.5;
  c.R2 = (float)(R * R);
  c.NR = (float)-R;
  c.N2R = (float)(-2.0 * R);
  c.S = (g.R0 - R) * (g.R0 + R);
  c.R0i = (int)fl;
  c.K1 = K1;
  c.mc = 0.5f - K0 - K1 - 1e-6f;
  return c;
}

// The correctly rounded fallback of the exact path, out of line: about one near pair in 2,000 needs it,
// and inlined its FP64 divide and square root cost the counting loop registers and instruction cache.
__device__ __noinline__ uint32_t ref_bin_slow(double d2, double bin, double inv_bin, double margin, uint32_t nhist) {
  return ref_bin(d2, bin, inv_bin, margin, nhist);
}

template <bool SAME, bool WINDOW, bool CENTRED, bool INWIN = false>
__device__ __forceinline__ unsigned count_tile_pair_t(const HistParams &p, const TilePair tp, const PairGeom &g,
                                                      uint8_t *stage, uint32_t *win, uint32_t base,
                                                      unsigned long long *h) {
  double *wI = reinterpret_cast<double *>(stage);
  // I rows in pairs (2p, 2p + 1), 8 floats a pair: x x' y y' z z' w w' (offsets; w = P_i, centred), so
  // that two 16-byte loads give both rows' values as packed pairs
  float *wIf = reinterpret_cast<float *>(wI + 3 * TILE_MAX);
  float4 *wI4 = reinterpret_cast<float4 *>(wIf);
  uint32_t *queue = reinterpret_cast<uint32_t *>(wI4 + TILE_MAX);
  const uint32_t lane = threadIdx.x & 31;
  const Tile TI = p.tiles[tp.I], TJ = p.tiles[tp.J];
  const uint32_t ni = TI.count, nj = TJ.count;
  const double ib = p.inv_bin;
  double cI[3], cJ[3];
  float dh[3], dl[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    cI[k] = 0.5 * (TI.lo[k] + TI.hi[k]);
    cJ[k] = 0.5 * (TJ.lo[k] + TJ.hi[k]);
    dh[k] = (float)g.D[k];
    dl[k] = (float)(g.D[k] - (double)dh[k]);
  }
  const float MAGIC = 12582912.0f;  // 1.5 * 2^23
  const uint32_t W = p.win;
  // Slots below Wl are window slots of bins below the last one and below 2^22 (the last bin and beyond,
  // and distances the magic-number rounding does not cover, take the exact path).  A slot computed
  // from r >= 2^22 is at least 2^22 - base: never below Wl.
  const uint32_t lim = min(p.nhist - 1u, 1u << 22);
  const uint32_t Wl = lim > base ? min(WINDOW ? W : 0xffffffffu, lim - base) : 0u;
  float m0 = 0.f, mr = 0.f;
  int tbase;
  CentredConsts cc;
  if (CENTRED) {
    cc = centred_consts(g);
    tbase = __float_as_int(MAGIC) + (int)base - cc.R0i;  // slot = bits(t + MAGIC) - tbase
  } else {
    const float Dm = (float)fmax(fabs(g.D[0]), fmax(fabs(g.D[1]), fabs(g.D[2])));
    m0 = 2.02f * (5.9604645e-8f * (2.0f * g.EI + 3.0f * g.EJ + 2.0f) + 9.094947e-13f * Dm) + 1e-6f;
    mr = 6.0f * 5.9604645e-8f;
    tbase = __float_as_int(MAGIC) + (int)base;  // slot = bits(r + MAGIC) - tbase - (d < 0)
  }
  for (uint32_t i = lane; i < ni; i += 32) {
    const double x = p.X[TI.start + i], y = p.Y[TI.start + i], z = p.Z[TI.start + i];
    wI[i] = x;
    wI[TILE_MAX + i] = y;
    wI[2 * TILE_MAX + i] = z;
    const double ax = (x - cI[0]) * ib, ay = (y - cI[1]) * ib, az = (z - cI[2]) * ib;
    float P = 0.f;
    if (CENTRED) P = (float)(2.0 * (g.D[0] * ax + g.D[1] * ay + g.D[2] * az) + (ax * ax + ay * ay + az * az) + cc.S);
    float *row = wIf + (i >> 1) * 8 + (i & 1);
    row[0] = (float)ax;
    row[2] = (float)ay;
    row[4] = (float)az;
    row[6] = P;
  }
  // Apart from a tile against itself, a pair's validity is not tested per pair: rows past the tile in
  // its last step and J slots past the tile hold NaN, so their estimates are never fast (every
  // comparison with NaN is false) and add 1 to the lane's spare slot; their near bits are dropped
  // once per step (cmask and the row mask below).
  if (!SAME && ni + lane < ((ni + 3u) & ~3u)) {
    float *row = wIf + ((ni + lane) >> 1) * 8 + ((ni + lane) & 1);
    row[0] = row[2] = row[4] = row[6] = __int_as_float(0x7fffffff);
  }
  const uint32_t j0 = lane, j1 = lane + 32;
  const bool c0 = j0 < nj, c1 = j1 < nj;
  // the J tile stays in registers: FP64 for the exact path (other lanes fetch it by shuffle), FP32
  // for the estimate
  double Xj0 = 0.0, Yj0 = 0.0, Zj0 = 0.0, Xj1 = 0.0, Yj1 = 0.0, Zj1 = 0.0;
  if (c0) {
    Xj0 = p.X[TJ.start + j0];
    Yj0 = p.Y[TJ.start + j0];
    Zj0 = p.Z[TJ.start + j0];
  }
  if (c1) {
    Xj1 = p.X[TJ.start + j1];
    Yj1 = p.Y[TJ.start + j1];
    Zj1 = p.Z[TJ.start + j1];
  }
  float xj0, yj0, zj0, xj1, yj1, zj1, qj0 = 0.f, qj1 = 0.f;
  {
    const double bx0 = (Xj0 - cJ[0]) * ib, by0 = (Yj0 - cJ[1]) * ib, bz0 = (Zj0 - cJ[2]) * ib;
    const double bx1 = (Xj1 - cJ[0]) * ib, by1 = (Yj1 - cJ[1]) * ib, bz1 = (Zj1 - cJ[2]) * ib;
    if (CENTRED) {  // -2 b rounded (the factor is exact) and Q_j
      xj0 = -2.0f * (float)bx0;
      yj0 = -2.0f * (float)by0;
      zj0 = -2.0f * (float)bz0;
      xj1 = -2.0f * (float)bx1;
      yj1 = -2.0f * (float)by1;
      zj1 = -2.0f * (float)bz1;
      qj0 = (float)(2.0 * (g.D[0] * bx0 + g.D[1] * by0 + g.D[2] * bz0) - (bx0 * bx0 + by0 * by0 + bz0 * bz0));
      qj1 = (float)(2.0 * (g.D[0] * bx1 + g.D[1] * by1 + g.D[2] * bz1) - (bx1 * bx1 + by1 * by1 + bz1 * bz1));
    } else {
      xj0 = (float)bx0 - dl[0];
      yj0 = (float)by0 - dl[1];
      zj0 = (float)bz0 - dl[2];
      xj1 = (float)bx1 - dl[0];
      yj1 = (float)by1 - dl[1];
      zj1 = (float)bz1 - dl[2];
    }
    if (!SAME) {
      const float nan = __int_as_float(0x7fffffff);
      if (!c0) xj0 = yj0 = zj0 = qj0 = nan;
      if (!c1) xj1 = yj1 = zj1 = qj1 = nan;
    }
  }
  // the J atoms' values and the tile pair's constants as packed pairs (both halves equal)
  using xns_f2::splat;
  const xns_f2::f2 XJ0 = splat(xj0), YJ0 = splat(yj0), ZJ0 = splat(zj0), XJ1 = splat(xj1), YJ1 = splat(yj1),
                   ZJ1 = splat(zj1), MAGIC2 = splat(MAGIC);
  xns_f2::f2 QJ0 = 0, QJ1 = 0, R2_2 = 0, NR2 = 0, N2R2 = 0, NK1_2 = 0, MC2 = 0;
  xns_f2::f2 DH0 = 0, DH1 = 0, DH2 = 0, MR2 = 0, M02 = 0;
  const xns_f2::f2 HALF2 = splat(0.5f), SIGN2 = 0x8000000080000000ull;  // SIGN2: flips both signs
  if (!CENTRED) {
    DH0 = splat(dh[0]);
    DH1 = splat(dh[1]);
    DH2 = splat(dh[2]);
    MR2 = splat(mr);
    M02 = splat(m0);
  }
  if (CENTRED) {
    QJ0 = splat(qj0);
    QJ1 = splat(qj1);
    R2_2 = splat(cc.R2);
    NR2 = splat(cc.NR);
    N2R2 = splat(cc.N2R);
    NK1_2 = splat(-cc.K1);
    MC2 = splat(cc.mc);
  }
  __syncwarp();
  const uint32_t below = (1u << lane) - 1u;  // lanes below this one
  const uint32_t tbase4 = (uint32_t)tbase * 4u, Wl4 = Wl * 4u, spare4 = (W + lane) * 4u;  // byte offsets
  const double nhm1 = (double)p.nhist - 1.0;
  uint32_t qn = 0, qd = 0;  // entries queued / binned (warp-uniform)
  unsigned bad = 0;
  // Lane l bins the pairs of queued entry qd + l exactly (l < n), then n entries are done.  An entry is
  // one lane's near pairs of one step: rows i .. i + 3 against that lane's J atoms (lane, lane + 32),
  // bit k of the mask standing for row i + k / 2 and J atom lane + 32 (k & 1).  The warp drains full
  // batches of 32 while it counts, so every lane has an entry.  The entries were stored by other lanes:
  // __syncwarp orders those stores before the loads.
  auto drain = [&](uint32_t n) {
    __syncwarp();
    const uint32_t e = lane < n ? queue[(qd + lane) & (QUEUE - 1)] : 0u;
    const uint32_t src = (e >> 8) & 31u, row = (e >> 13) << 2;
    uint32_t pm = e & 255u;
    // the J atoms sit in lane src
    const double xb0 = __shfl_sync(0xffffffffu, Xj0, src), xb1 = __shfl_sync(0xffffffffu, Xj1, src);
    const double yb0 = __shfl_sync(0xffffffffu, Yj0, src), yb1 = __shfl_sync(0xffffffffu, Yj1, src);
    const double zb0 = __shfl_sync(0xffffffffu, Zj0, src), zb1 = __shfl_sync(0xffffffffu, Zj1, src);
    while (pm) {
      const uint32_t bit = __ffs(pm) - 1;
      pm &= pm - 1;
      const uint32_t a = row + (bit >> 1);
      const bool hi = (bit & 1u) != 0;
      const double d2 = ref_dist2(wI[a], wI[TILE_MAX + a], wI[2 * TILE_MAX + a], hi ? xb1 : xb0, hi ? yb1 : yb0,
                                  hi ? zb1 : zb0);
      uint32_t k;
      if (!ref_bin_fast(d2, p.inv_bin, p.margin, nhm1, &k)) k = ref_bin_slow(d2, p.bin, p.inv_bin, p.margin, p.nhist);
      if (k >= p.nhist) {
        bad++;
      } else if (WINDOW && k - base < W) {
        atomicAdd(win + (k - base), 1u);
      } else {
        atomicAdd(h + k, 1ull);
      }
    }
    qd += n;
  };
  // FAST: the estimate's bin is certain and its slot is below Wl; a lane without a fast pair adds 1 to
  // its own spare slot instead (branch-free; the 32 spare slots are never flushed or read), near pairs
  // set their bit K of the step's mask.  Slots are byte offsets (4 x the bin's slot, modulo 2^32): a
  // slot of a valid pair lies within +-2^23, so the unsigned test against 4 Wl keeps its meaning.
#define XNS_COUNT(FAST, SLOT, VALID, K, NM)                                                 \
  {                                                                                         \
    const bool fast = (VALID) && (FAST) && (INWIN || (SLOT) < Wl4);                         \
    if (WINDOW) {                                                                           \
      atomicAdd(reinterpret_cast<uint32_t *>(reinterpret_cast<char *>(win) + (fast ? (SLOT) : spare4)), 1u); \
    } else if (fast) {                                                                      \
      atomicAdd(h + ((SLOT) >> 2), 1ull);                                                   \
    }                                                                                       \
    NM |= ((VALID) && !fast) ? (1u << (K)) : 0u;                                            \
  }
// The direct estimate for two pairs at once (rows i, i + 1 against one J atom), packed: per half, the
// scalar operations dx = dh + (x_i - x_j) (each axis), d2 by FMAs, r0 = d2 rsqrt(d2), one Newton
// step, the magic-number rounding, in that order.
#define XNS_DIRECT2(RX, RY, RZ, XJ, YJ, ZJ, VLO, VHI, KLO, KHI, NM)                          \
  {                                                                                         \
    using namespace xns_f2;                                                                 \
    const f2 dx = add(DH0, sub(RX, XJ)), dy = add(DH1, sub(RY, YJ)), dz = add(DH2, sub(RZ, ZJ)); \
    const f2 d2 = xns_f2::fma(dx, dx, xns_f2::fma(dy, dy, mul(dz, dz)));                    \
    float y0, y1;                                                                           \
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y0) : "f"(lo(d2)));                           \
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y1) : "f"(hi(d2)));                           \
    const f2 y = pack(y0, y1);                                                              \
    const f2 r0 = mul(d2, y); /* NaN for d2 == 0: not fast */                               \
    const f2 r = xns_f2::fma(xns_f2::fma(r0 ^ SIGN2, r0, d2), mul(HALF2, y), r0);           \
    const f2 t = add(r, MAGIC2);                                                            \
    const f2 d = sub(r, sub(t, MAGIC2));                                                    \
    const f2 m = xns_f2::fma(r, MR2, M02);                                                  \
    const uint32_t slo = (uint32_t)__float_as_int(lo(t)) * 4u - tbase4 - (lo(d) < 0.f ? 4u : 0u); \
    const uint32_t shi = (uint32_t)__float_as_int(hi(t)) * 4u - tbase4 - (hi(d) < 0.f ? 4u : 0u); \
    XNS_COUNT(fabsf(lo(d)) >= lo(m), slo, VLO, KLO, NM)                                     \
    XNS_COUNT(fabsf(hi(d)) >= hi(m), shi, VHI, KHI, NM)                                     \
  }
#define XNS_CENTRED2(RX, RY, RZ, RW, XJ, YJ, ZJ, QJ, VLO, VHI, KLO, KHI, NM)                \
  {                                                                                         \
    using namespace xns_f2;                                                                 \
    const f2 num = add(sub(RW, QJ), xns_f2::fma(RX, XJ, xns_f2::fma(RY, YJ, mul(RZ, ZJ)))); \
    const f2 d2 = add(num, R2_2);                                                           \
    float y0, y1;                                                                           \
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y0) : "f"(lo(d2)));                           \
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y1) : "f"(hi(d2)));                           \
    const f2 y = pack(y0, y1);                                                              \
    const f2 t0 = xns_f2::fma(d2, y, NR2);                      /* r - R, to ~5u r */       \
    const f2 res = xns_f2::fma(t0, sub(N2R2, t0), num);         /* num - t0 (t0 + 2R) */    \
    const f2 t = xns_f2::fma(res, mul(y, HALF2), t0);           /* r - floor(R0) - 0.5 */   \
    const f2 tm = add(t, MAGIC2);                                                           \
    const f2 d = sub(t, sub(tm, MAGIC2));                                                   \
    const f2 m = xns_f2::fma(xns_f2::abs(t), NK1_2, MC2);                                   \
    const uint32_t slo = (uint32_t)__float_as_int(lo(tm)) * 4u - tbase4;                   \
    const uint32_t shi = (uint32_t)__float_as_int(hi(tm)) * 4u - tbase4;                   \
    XNS_COUNT(fabsf(lo(d)) <= lo(m), slo, VLO, KLO, NM)                                     \
    XNS_COUNT(fabsf(hi(d)) <= hi(m), shi, VHI, KHI, NM)                                     \
  }
  // lanes with near pairs in the step's rows ROW .. ROW + 3 append one entry each, in lane order;
  // fewer than 32 entries wait between steps and a push adds at most 32: never more than 63 queued
#define XNS_PUSH(NM, ROW)                                                                   \
  {                                                                                         \
    const unsigned nb = __ballot_sync(0xffffffffu, NM != 0);                                \
    if (NM) queue[(qn + __popc(nb & below)) & (QUEUE - 1)] = (((ROW) >> 2) << 13) | (lane << 8) | NM; \
    qn += __popc(nb);                                                                       \
  }
  // a step: rows i .. i + 3 (two row pairs) against the lane's two J atoms.  A tile against itself
  // tests validity per pair (i < j, both inside the tile); other tile pairs rely on the NaN padding.
  const uint32_t cmask = (c0 ? 0x55u : 0u) | (c1 ? 0xAAu : 0u);  // near bits of the lane's real J atoms
  for (uint32_t i = 0; i < ni; i += 4) {
    const float4 pa = wI4[i], pb = wI4[i + 1], pc = wI4[i + 2], pd = wI4[i + 3];  // (x x' y y'), (z z' w w')
    bool va0 = true, va1 = true, vb0 = true, vb1 = true, vc0 = true, vc1 = true, vd0 = true, vd1 = true;
    if (SAME) {
      va0 = c0;
      va1 = c1;
      vb0 = c0 && i + 1 < ni;
      vb1 = c1 && i + 1 < ni;
      vc0 = c0 && i + 2 < ni;
      vc1 = c1 && i + 2 < ni;
      vd0 = c0 && i + 3 < ni;
      vd1 = c1 && i + 3 < ni;
      va0 = va0 && i < j0;
      va1 = va1 && i < j1;
      vb0 = vb0 && i + 1 < j0;
      vb1 = vb1 && i + 1 < j1;
      vc0 = vc0 && i + 2 < j0;
      vc1 = vc1 && i + 2 < j1;
      vd0 = vd0 && i + 3 < j0;
      vd1 = vd1 && i + 3 < j1;
    }
    // near pairs of the row pairs (i, i + 1) and (i + 2, i + 3): bit k is row + k / 2, J atom lane + 32 (k & 1)
    uint32_t nmA = 0, nmB = 0;
    if (CENTRED) {
      using xns_f2::pack;
      const xns_f2::f2 XA = pack(pa.x, pa.y), YA = pack(pa.z, pa.w), ZA = pack(pb.x, pb.y), WA = pack(pb.z, pb.w);
      const xns_f2::f2 XB = pack(pc.x, pc.y), YB = pack(pc.z, pc.w), ZB = pack(pd.x, pd.y), WB = pack(pd.z, pd.w);
      XNS_CENTRED2(XA, YA, ZA, WA, XJ0, YJ0, ZJ0, QJ0, va0, vb0, 0, 2, nmA)
      XNS_CENTRED2(XA, YA, ZA, WA, XJ1, YJ1, ZJ1, QJ1, va1, vb1, 1, 3, nmA)
      XNS_CENTRED2(XB, YB, ZB, WB, XJ0, YJ0, ZJ0, QJ0, vc0, vd0, 0, 2, nmB)
      XNS_CENTRED2(XB, YB, ZB, WB, XJ1, YJ1, ZJ1, QJ1, vc1, vd1, 1, 3, nmB)
    } else {
      using xns_f2::pack;
      const xns_f2::f2 XA = pack(pa.x, pa.y), YA = pack(pa.z, pa.w), ZA = pack(pb.x, pb.y);
      const xns_f2::f2 XB = pack(pc.x, pc.y), YB = pack(pc.z, pc.w), ZB = pack(pd.x, pd.y);
      XNS_DIRECT2(XA, YA, ZA, XJ0, YJ0, ZJ0, va0, vb0, 0, 2, nmA)
      XNS_DIRECT2(XA, YA, ZA, XJ1, YJ1, ZJ1, va1, vb1, 1, 3, nmA)
      XNS_DIRECT2(XB, YB, ZB, XJ0, YJ0, ZJ0, vc0, vd0, 0, 2, nmB)
      XNS_DIRECT2(XB, YB, ZB, XJ1, YJ1, ZJ1, vc1, vd1, 1, 3, nmB)
    }
    uint32_t nm = nmA | (nmB << 4);  // bit k: row i + k / 2, J atom lane + 32 (k & 1)
    if (!SAME) {  // drop the NaN pairs: rows ni and beyond, J slots past the tile
      const uint32_t v = ni - i;
      nm &= cmask & (v >= 4 ? 0xFFu : (1u << (2 * v)) - 1u);
    }
    XNS_PUSH(nm, i)
    while (qn - qd >= 32) drain(32);
  }
#undef XNS_PUSH
#undef XNS_CENTRED2
#undef XNS_DIRECT2
#undef XNS_COUNT
  if (qn != qd) drain(qn - qd);
  __syncwarp();  // every lane is done with the stage before the warp's next tile pair refills it
  return bad;
}

template <bool WINDOW>
__device__ __forceinline__ unsigned count_tile_pair(const HistParams &p, const TilePair tp, uint8_t *stage, uint32_t *win,
                                                    uint32_t base, unsigned long long *h) {
  const PairGeom g = pair_geom(p.tiles[tp.I], p.tiles[tp.J], p.inv_bin);
  if (tp.I == tp.J) return count_tile_pair_t<true, WINDOW, false>(p, tp, g, stage, win, base, h);
  if (far_pair(g)) {
    // Every bin the tile pair can reach ([kmin, kmax], from the tiles' boxes, at or above the window's
    // base inside a run) lies in the window and below the last bin and 2^22: the slot of a fast pair,
    // its exact bin - base, needs no test (INWIN).
    if (WINDOW && tp.kmax < min(base + p.win, min(p.nhist - 1u, 1u << 22)))
      return count_tile_pair_t<false, WINDOW, true, true>(p, tp, g, stage, win, base, h);
    return count_tile_pair_t<false, WINDOW, true>(p, tp, g, stage, win, base, h);
  }
  return count_tile_pair_t<false, WINDOW, false>(p, tp, g, stage, win, base, h);
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

// Moves the window of W bins from B to nb > B: bins [B, nb) leave (flushed), bins [nb, B + W) move
// down to slots [0, B + W - nb), the vacated top slots are cleared.  Called by all threads between
// barriers.
__device__ __forceinline__ void slide_window(uint32_t *win, uint32_t W, unsigned long long *h, uint32_t B, uint32_t nb,
                                             uint32_t nhist) {
  const uint32_t delta = nb - B;
  flush_window(win, h, B, 0, min(delta, W), nhist);
  if (delta >= W) return;  // everything left; the flush cleared it
  __syncthreads();
  // shift down by delta in chunks: a chunk's reads lie above every slot written so far
  for (uint32_t c = 0; c < W - delta; c += HW_THREADS) {
    const uint32_t s = c + threadIdx.x;
    const uint32_t v = s < W - delta ? win[s + delta] : 0u;
    __syncthreads();
    if (s < W - delta) win[s] = v;
    __syncthreads();
  }
  for (uint32_t s = W - delta + threadIdx.x; s < W; s += HW_THREADS) win[s] = 0;
}

// Persistent: each CTA takes runs (one class, a contiguous stretch of the sorted list) from the queue.
// The window is empty between runs (the final flush clears every slot below nhist, and slots at or
// above nhist are never written).
__global__ void __launch_bounds__(HW_THREADS, 1) hist_window_kernel(HistParams p) {
  extern __shared__ uint32_t win[];  // p.win bins, 32 spare slots, then WARP_STAGE bytes per warp
  const uint32_t W = p.win;
  uint8_t *stage = reinterpret_cast<uint8_t *>(win + W + 32) + (threadIdx.x >> 5) * WARP_STAGE;
  __shared__ uint32_t run;
  for (uint32_t s = threadIdx.x; s < W; s += HW_THREADS) win[s] = 0;
  unsigned bad = 0;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) run = atomicAdd(p.queue, 1u);
    __syncthreads();
    const uint32_t ri = run;
    if (ri >= p.nranges) break;
    const CtaRange rg = p.ranges[ri];
    unsigned long long *h = p.hist + (size_t)rg.type * p.nhist;
    uint32_t B = p.list[rg.begin].kmin / BUCKET * BUCKET;
    for (uint32_t r = rg.begin; r < rg.end; r += HW_WARPS) {
      // the round's entries must fit the window [B, B + W): slide it when the farthest one does not
      uint32_t kmax = 0;
      for (uint32_t e = r; e < min(r + HW_WARPS, rg.end); e++) kmax = max(kmax, p.list[e].kmax);
      if (kmax >= B + W) {
        const uint32_t nb = p.list[r].kmin / BUCKET * BUCKET;
        if (nb > B) {
          __syncthreads();
          slide_window(win, W, h, B, nb, p.nhist);
          B = nb;
          __syncthreads();
        }
      }
      const uint32_t e = r + (threadIdx.x >> 5);
      if (e < rg.end) {
        bad += count_tile_pair<true>(p, p.list[e], stage, win, B, h);
      }
    }
    __syncthreads();
    flush_window(win, h, B, 0, W, p.nhist);
  }
  if (bad) atomicAdd(p.n_bad, bad);
}

__global__ void __launch_bounds__(256, 2) hist_wide_kernel(HistParams p) {
  __shared__ __align__(16) uint8_t stage_all[8 * WARP_STAGE];
  uint8_t *stage = stage_all + (threadIdx.x >> 5) * WARP_STAGE;
  unsigned bad = 0;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t e = p.wide_begin + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); e < p.wide_end; e += nw) {
    const TilePair tp = p.list[e];
    const ElemCls ea = p.ecls[p.tiles[tp.I].elem], eb = p.ecls[p.tiles[tp.J].elem];
    const uint32_t a = min(ea.local, eb.local), b = max(ea.local, eb.local), n = ea.nel_s;
    unsigned long long *h = p.hist + (size_t)(ea.cls_base + a * n - a * (a - 1) / 2 + (b - a)) * p.nhist;
    bad += count_tile_pair<false>(p, tp, stage, nullptr, 0, h);
  }
  if (bad) atomicAdd(p.n_bad, bad);
}

}  // namespace

int xns_hist_plan(xns_ctx *ctx, const HistSet &hs, uint32_t nhist, double bin, unsigned long long *d_hist,
                  const HistTuning &tune, HistLaunch *L) {
  const uint32_t nel = (uint32_t)hs.el_n.size();
  *L = HistLaunch();
  if (nhist == 0 || !(bin > 0)) return xns_fail(ctx, XNS_ERR_ARG, "histogram: nhist == 0 or bin <= 0");
  if (nel == 0) return xns_fail(ctx, XNS_ERR_ARG, "histogram: no elements");
  if (tune.win < 2 * BUCKET || tune.win > WIN_MAX || tune.win % 4 || tune.cell_target < 8)
    return xns_fail(ctx, XNS_ERR_ARG, "histogram: tuning outside its range");
  if (tune.nshard == 0 || tune.shard >= tune.nshard) return xns_fail(ctx, XNS_ERR_ARG, "histogram: shard >= nshard");
  // classes: structure s owns P(nel_s) consecutive classes
  std::vector<ElemCls> ecls(nel);
  uint32_t C = 0;
  for (const HistStruct &s : hs.st) {
    for (uint32_t l = 0; l < s.nel; l++) ecls[s.e0 + l] = {C, l, s.nel, 0};
    C += xns_npairs(s.nel);
  }
  int st;
  void *flags;
  if ((st = xns_scratch(ctx, SLOT_HFLAGS, 64, &flags))) return st;
  L->hist = d_hist;
  L->hist_words = (size_t)C * nhist;
  L->flags = (unsigned int *)flags;
  L->classes = C;
  uint32_t ntot = 0;
  for (uint32_t e = 0; e < nel; e++) ntot = std::max(ntot, hs.el_off[e] + hs.el_n[e]);
  if (ntot < 2) return XNS_OK;

  // -- element bounding boxes -> cell grids
  void *vaux, *vh;
  const size_t aux_bytes = (sizeof(ElemGrid) + sizeof(ElemCls) + 6 * sizeof(unsigned long long) + 2 * sizeof(uint32_t)) * nel + 64;
  if ((st = xns_scratch(ctx, SLOT_AUX, aux_bytes, &vaux))) return st;
  ElemGrid *d_eg = (ElemGrid *)vaux;
  ElemCls *d_ecls = (ElemCls *)(d_eg + nel);
  unsigned long long *d_bmin = (unsigned long long *)(d_ecls + nel), *d_bmax = d_bmin + 3 * nel;
  uint32_t *d_ebase = (uint32_t *)(d_bmax + 3 * nel), *d_estart = d_ebase + nel;
  if ((st = xns_pinned(ctx, aux_bytes, &vh))) return st;
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  std::vector<ElemGrid> eg(nel);
  for (uint32_t e = 0; e < nel; e++) {
    memset(&eg[e], 0, sizeof(ElemGrid));
    eg[e].atom0 = hs.el_off[e];
    eg[e].natoms = hs.el_n[e];
  }
  memcpy(vh, eg.data(), sizeof(ElemGrid) * nel);
  memcpy((char *)vh + sizeof(ElemGrid) * nel, ecls.data(), sizeof(ElemCls) * nel);
  XNS_CUDA(ctx, cudaMemcpyAsync(d_eg, vh, (sizeof(ElemGrid) + sizeof(ElemCls)) * nel, cudaMemcpyHostToDevice, ctx->stream));
  XNS_CUDA(ctx, cudaMemsetAsync(d_bmin, 0xff, 3 * sizeof(unsigned long long) * nel, ctx->stream));
  XNS_CUDA(ctx, cudaMemsetAsync(d_bmax, 0, 3 * sizeof(unsigned long long) * nel, ctx->stream));
  elem_bbox_kernel<<<dim3(std::max(1, ctx->num_sms / (int)nel), nel), 256, 0, ctx->stream>>>(hs.x, hs.y, hs.z, d_eg, d_bmin,
                                                                                             d_bmax);
  XNS_LAUNCHED(ctx);
  std::vector<unsigned long long> bb(6 * (size_t)nel);
  XNS_CUDA(ctx, cudaMemcpyAsync(bb.data(), d_bmin, 6 * sizeof(unsigned long long) * nel, cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  uint32_t ncells = 0, ccells = 0;
  std::vector<uint32_t> ebase(nel);
  std::vector<ElemGrid> cand((size_t)nel * NCAND);
  for (uint32_t e = 0; e < nel; e++) {
    ElemGrid &g = eg[e];
    g.base = 0;
    for (int c = 0; c < NCAND; c++) {
      cand[(size_t)e * NCAND + c] = g;
      cand[(size_t)e * NCAND + c].n[0] = cand[(size_t)e * NCAND + c].n[1] = cand[(size_t)e * NCAND + c].n[2] = 0;
    }
    if (!g.natoms) continue;
    double ext[3], vol = 1;
    for (int k = 0; k < 3; k++) {
      g.o[k] = ord_value(bb[3 * e + k]);
      ext[k] = ord_value(bb[3 * (size_t)nel + 3 * e + k]) - g.o[k];
      if (!(ext[k] >= 0) || !std::isfinite(ext[k])) return xns_fail(ctx, XNS_ERR_ARG, "histogram: non-finite coordinates");
    }
    const double emax = std::max(ext[0], std::max(ext[1], ext[2]));
    for (int k = 0; k < 3; k++) vol *= std::max(ext[k], 1e-3 * emax + 1e-9);
    const double s = std::max(cbrt(tune.cell_target * vol / g.natoms), 1e-6);
    // candidates: the grid of cell edge s, and grids whose cells divide the extent evenly for edges
    // near s (a grid that leaves a thin layer of part-empty cells wastes lanes on small tiles)
    static const double scale[NCAND - 1] = {0.88, 0.94, 1.0, 1.06, 1.12};
    for (int c = 0; c < NCAND; c++) {
      ElemGrid &q = cand[(size_t)e * NCAND + c];
      q = g;
      q.base = ccells;
      for (int k = 0; k < 3; k++) {
        const double n = c == 0 ? floor(ext[k] / s) + 1 : round(ext[k] / (s * scale[c - 1]));
        q.n[k] = (uint32_t)std::min<double>(MAX_CELLS_AXIS, std::max(1.0, n));
        q.inv[k] = ext[k] > 0 ? q.n[k] / (ext[k] * (1 + 1e-12)) : 0.0;
      }
      ccells += q.n[0] * q.n[1] * q.n[2];
    }
  }
  // -- per element, the candidate grid whose tiles occupy the fewest lanes (cells no larger than the
  // largest candidate's), counted on the device
  {
    void *vcand, *vslots;
    if ((st = xns_scratch(ctx, SLOT_HCELL, sizeof(uint32_t) * (size_t)ccells + 64, &vcand))) return st;
    if ((st = xns_scratch(ctx, SLOT_HKEY, (sizeof(ElemGrid) + sizeof(unsigned long long)) * cand.size() + 64, &vslots)))
      return st;
    ElemGrid *d_cg = (ElemGrid *)vslots;
    unsigned long long *d_slots = (unsigned long long *)(d_cg + cand.size());
    void *vh2;
    if ((st = xns_pinned(ctx, std::max(aux_bytes, (sizeof(ElemGrid) + sizeof(unsigned long long)) * cand.size()), &vh2)))
      return st;
    memcpy(vh2, cand.data(), sizeof(ElemGrid) * cand.size());
    XNS_CUDA(ctx, cudaMemcpyAsync(d_cg, vh2, sizeof(ElemGrid) * cand.size(), cudaMemcpyHostToDevice, ctx->stream));
    XNS_CUDA(ctx, cudaMemsetAsync(vcand, 0, sizeof(uint32_t) * (size_t)ccells, ctx->stream));
    XNS_CUDA(ctx, cudaMemsetAsync(d_slots, 0, sizeof(unsigned long long) * cand.size(), ctx->stream));
    cand_count_kernel<<<dim3(std::max(1, ctx->num_sms / (int)nel), nel, NCAND), 256, 0, ctx->stream>>>(
        hs.x, hs.y, hs.z, d_cg, (uint32_t *)vcand);
    XNS_LAUNCHED(ctx);
    cand_slots_kernel<<<(unsigned)cand.size(), 256, 0, ctx->stream>>>((const uint32_t *)vcand, d_cg, d_slots);
    XNS_LAUNCHED(ctx);
    std::vector<unsigned long long> slots(cand.size());
    XNS_CUDA(ctx, cudaMemcpyAsync(slots.data(), d_slots, sizeof(unsigned long long) * cand.size(),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (uint32_t e = 0; e < nel; e++) {
      if (!eg[e].natoms) continue;
      int best = 0;
      for (int c = 1; c < NCAND; c++)
        if (slots[(size_t)e * NCAND + c] < slots[(size_t)e * NCAND + best]) best = c;
      const ElemGrid &q = cand[(size_t)e * NCAND + best];
      for (int k = 0; k < 3; k++) {
        eg[e].n[k] = q.n[k];
        eg[e].inv[k] = q.inv[k];
      }
    }
    for (uint32_t e = 0; e < nel; e++) {
      eg[e].base = ncells;
      if (eg[e].natoms) ncells += eg[e].n[0] * eg[e].n[1] * eg[e].n[2];
    }
    vh = vh2;  // the pinned staging buffer may have moved
  }

  // -- counting sort of atoms by cell
  void *vcell, *vsort;
  if ((st = xns_scratch(ctx, SLOT_HCELL, sizeof(uint32_t) * (4 * (size_t)ncells + 8), &vcell))) return st;
  uint32_t *d_cnt = (uint32_t *)vcell, *d_coff = d_cnt + ncells, *d_toff = d_coff + ncells, *d_cur = d_toff + ncells,
           *d_tot = d_cur + ncells;
  const bool ordered = tune.nshard > 1 || tune.ordered;
  if ((st = xns_scratch(ctx, SLOT_HSORT, (sizeof(double) * 3 + sizeof(uint32_t) * (ordered ? 2 : 1)) * (size_t)ntot,
                        &vsort)))
    return st;
  double *Xs = (double *)vsort, *Ys = Xs + ntot, *Zs = Ys + ntot;
  uint32_t *d_cid = (uint32_t *)(Zs + ntot), *d_idx = ordered ? d_cid + ntot : nullptr;
  for (uint32_t e = 0; e < nel; e++) ebase[e] = std::min(eg[e].base, ncells - 1);
  memcpy(vh, eg.data(), sizeof(ElemGrid) * nel);
  memcpy((char *)vh + sizeof(ElemGrid) * nel, ebase.data(), sizeof(uint32_t) * nel);
  XNS_CUDA(ctx, cudaMemcpyAsync(d_eg, vh, sizeof(ElemGrid) * nel, cudaMemcpyHostToDevice, ctx->stream));
  XNS_CUDA(ctx, cudaMemcpyAsync(d_ebase, (char *)vh + sizeof(ElemGrid) * nel, sizeof(uint32_t) * nel,
                                cudaMemcpyHostToDevice, ctx->stream));
  XNS_CUDA(ctx, cudaMemsetAsync(d_cnt, 0, sizeof(uint32_t) * ncells, ctx->stream));
  XNS_CUDA(ctx, cudaMemsetAsync(d_cur, 0, sizeof(uint32_t) * ncells, ctx->stream));
  const int gx = std::max(1, ctx->num_sms * 4 / (int)nel);
  cell_count_kernel<<<dim3(gx, nel), 256, 0, ctx->stream>>>(hs.x, hs.y, hs.z, d_eg, d_cid, d_cnt);
  XNS_LAUNCHED(ctx);
  scan_kernel<<<1, SCAN_THREADS, 0, ctx->stream>>>(d_cnt, ncells, d_coff, d_toff, d_tot);
  XNS_LAUNCHED(ctx);
  cell_scatter_kernel<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(hs.x, hs.y, hs.z, ntot, d_cid, d_coff, d_cur, Xs, Ys, Zs,
                                                                  d_idx);
  XNS_LAUNCHED(ctx);
  if (ordered) {
    cell_order_kernel<<<(ncells + 127) / 128, 128, 0, ctx->stream>>>(ncells, d_coff, d_cnt, Xs, Ys, Zs, d_idx);
    XNS_LAUNCHED(ctx);
  }
  // tiles per element: the tile offsets at the element boundaries
  gather_u32_kernel<<<(nel + 255) / 256, 256, 0, ctx->stream>>>(d_toff, d_ebase, nel, d_estart);
  XNS_LAUNCHED(ctx);
  std::vector<uint32_t> tstart(nel + 1);
  uint32_t totals[2];
  XNS_CUDA(ctx, cudaMemcpyAsync(totals, d_tot, sizeof(totals), cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaMemcpyAsync(tstart.data(), d_estart, sizeof(uint32_t) * nel, cudaMemcpyDeviceToHost, ctx->stream));
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

  // -- tile pairs sorted by (class, distance bucket)
  std::vector<Segment> sa, sb;
  std::vector<uint32_t> cls, same;
  for (const HistStruct &s : hs.st) {
    uint32_t t = ecls[s.e0].cls_base;
    for (uint32_t a = s.e0; a < s.e0 + s.nel; a++)
      for (uint32_t b = a; b < s.e0 + s.nel; b++, t++) {
        sa.push_back({tstart[a], tstart[a + 1] - tstart[a]});
        sb.push_back({tstart[b], tstart[b + 1] - tstart[b]});
        cls.push_back(t);
        same.push_back(a == b);
      }
  }
  std::vector<SegPair> sched;
  const unsigned long long ntp_all = xns_build_schedule(sa, sb, cls, same, 1, 1, &sched);
  L->ntp_total = ntp_all;
  // this pass: tile pairs [w_begin, w_begin + ntp) of the enumeration
  unsigned long long ntp = ntp_all > tune.w_begin ? ntp_all - tune.w_begin : 0;
  if (tune.max_pairs) ntp = std::min(ntp, tune.max_pairs);
  if (ntp >= (1ull << 32)) return xns_fail(ctx, XNS_ERR_ARG, "histogram: too many tile pairs for one pass");
  if (ntp == 0) return XNS_OK;
  SegPair *d_sp;
  if ((st = xns_upload_schedule(ctx, sched, &d_sp))) return st;
  KeyParams kp;
  kp.sp = d_sp;
  kp.nsp = (int)sched.size();
  kp.ntp = ntp;
  kp.wbeg = tune.w_begin;
  kp.tiles = d_tiles;
  kp.inv_bin = 1.0 / bin;
  kp.nhist = nhist;
  kp.nbuckets = nhist / BUCKET + 1;
  const unsigned long long nkeys = (unsigned long long)C * kp.nbuckets + 1;
  if (nkeys >= (1ull << 31)) return xns_fail(ctx, XNS_ERR_ARG, "histogram: too many classes x distance buckets");
  kp.nkeys = (uint32_t)nkeys;
  kp.win = tune.win;
  kp.shard = tune.shard;
  kp.nshard = tune.nshard;
  void *vk, *vl;
  if ((st = xns_scratch(ctx, SLOT_HKEY, sizeof(uint32_t) * (3 * (size_t)kp.nkeys + 8), &vk))) return st;
  uint32_t *d_kcnt = (uint32_t *)vk, *d_koff = d_kcnt + kp.nkeys, *d_kcur = d_koff + kp.nkeys, *d_ktot = d_kcur + kp.nkeys;
  if ((st = xns_scratch(ctx, SLOT_HLIST, sizeof(TilePair) * ntp, &vl))) return st;
  TilePair *d_list = (TilePair *)vl;
  XNS_CUDA(ctx, cudaMemsetAsync(d_kcnt, 0, sizeof(uint32_t) * kp.nkeys, ctx->stream));
  XNS_CUDA(ctx, cudaMemsetAsync(d_kcur, 0, sizeof(uint32_t) * kp.nkeys, ctx->stream));
  const int kgrid = ctx->num_sms * 8;
  void *vt;
  if ((st = xns_scratch(ctx, SLOT_HTMP, (sizeof(TilePair) + sizeof(uint32_t)) * ntp, &vt))) return st;
  TilePair *d_tmp = (TilePair *)vt;
  uint32_t *d_tkey = (uint32_t *)(d_tmp + ntp);
  pair_key_kernel<<<kgrid, 256, 0, ctx->stream>>>(kp, d_kcnt, d_tmp, d_tkey);
  XNS_LAUNCHED(ctx);
  scan_kernel<<<1, SCAN_THREADS, 0, ctx->stream>>>(d_kcnt, kp.nkeys, d_koff, nullptr, d_ktot);
  XNS_LAUNCHED(ctx);
  pair_scatter_kernel<<<kgrid, 256, 0, ctx->stream>>>(kp, d_koff, d_kcur, d_tmp, d_tkey, d_list);
  XNS_LAUNCHED(ctx);
  // cut the sorted list into runs of one class: about 4 runs per SM over the whole list, so that the
  // queue balances uneven classes; a CTA's u32 window counts at most 64*64*entries pairs per bin, so a
  // run stays below 2^19 entries
  std::vector<uint32_t> koff(kp.nkeys);
  uint32_t n_list = 0;  // tile pairs in this plan's list: all of them, or this shard's share
  XNS_CUDA(ctx, cudaMemcpyAsync(koff.data(), d_koff, sizeof(uint32_t) * kp.nkeys, cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaMemcpyAsync(&n_list, d_ktot, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const uint32_t n_narrow = koff[kp.nkeys - 1];
  const uint32_t run_len =
      std::min<uint32_t>(1u << 19, std::max<uint32_t>(64, (n_narrow + 4 * ctx->num_sms - 1) / (4 * ctx->num_sms)));
  std::vector<CtaRange> ranges;
  for (uint32_t c = 0; c < C; c++) {
    const uint32_t b0 = koff[(size_t)c * kp.nbuckets], b1 = koff[(size_t)(c + 1) * kp.nbuckets];
    for (uint32_t s = b0; s < b1; s += run_len) ranges.push_back({s, std::min(b1, s + run_len), c, 0});
  }
  std::stable_sort(ranges.begin(), ranges.end(),
                   [](const CtaRange &a, const CtaRange &b) { return a.end - a.begin > b.end - b.begin; });
  HistParams hp;
  hp.X = Xs;
  hp.Y = Ys;
  hp.Z = Zs;
  hp.tiles = d_tiles;
  hp.list = d_list;
  hp.ecls = d_ecls;
  hp.queue = (unsigned int *)flags + 1;
  hp.hist = d_hist;
  hp.n_bad = (unsigned int *)flags;
  hp.bin = bin;
  hp.inv_bin = 1.0 / bin;
  hp.margin = (double)nhist * ldexp(1.0, -37);
  hp.nhist = nhist;
  hp.nranges = (uint32_t)ranges.size();
  hp.wide_begin = n_narrow;
  hp.wide_end = n_list;
  hp.ranges = nullptr;
  hp.win = tune.win;
  if (!ranges.empty()) {
    void *vr, *vrh;
    if ((st = xns_scratch(ctx, SLOT_SEGPAIRS, sizeof(CtaRange) * ranges.size() + sizeof(SegPair) * sched.size(), &vr)))
      return st;
    // the schedule is no longer needed once the list is built; its slot now holds the runs
    if ((st = xns_pinned(ctx, sizeof(CtaRange) * ranges.size(), &vrh))) return st;
    XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    memcpy(vrh, ranges.data(), sizeof(CtaRange) * ranges.size());
    XNS_CUDA(ctx, cudaMemcpyAsync(vr, vrh, sizeof(CtaRange) * ranges.size(), cudaMemcpyHostToDevice, ctx->stream));
    hp.ranges = (const CtaRange *)vr;
  }
  memcpy(L->params, &hp, sizeof(hp));
  L->nranges = (uint32_t)ranges.size();
  L->window_grid = (uint32_t)std::min<size_t>((size_t)ctx->num_sms, ranges.size());
  L->window_smem = sizeof(uint32_t) * (tune.win + 32) + (size_t)WARP_STAGE * HW_WARPS;
  L->wide = hp.wide_end > hp.wide_begin;
  return XNS_OK;
}

int xns_hist_enqueue(xns_ctx *ctx, const HistLaunch &L) {
  if (L.zero_hist) XNS_CUDA(ctx, cudaMemsetAsync(L.hist, 0, sizeof(unsigned long long) * L.hist_words, ctx->stream));
  XNS_CUDA(ctx, cudaMemsetAsync(L.flags, 0, 2 * sizeof(unsigned int), ctx->stream));
  HistParams hp;
  memcpy(&hp, L.params, sizeof(hp));
  if (L.nranges) {
    static bool attr[XNS_MAX_DEVICES] = {};  // the attribute is per device; set once on each
    if (ctx->device < 0 || ctx->device >= XNS_MAX_DEVICES || !attr[ctx->device]) {
      const int max_smem = (int)(sizeof(uint32_t) * (WIN_MAX + 32) + (size_t)WARP_STAGE * HW_WARPS);
      XNS_CUDA(ctx, cudaFuncSetAttribute(hist_window_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem));
      if (ctx->device >= 0 && ctx->device < XNS_MAX_DEVICES) attr[ctx->device] = true;
    }
    hist_window_kernel<<<L.window_grid, HW_THREADS, L.window_smem, ctx->stream>>>(hp);
    XNS_LAUNCHED(ctx);
  }
  if (L.wide) {
    hist_wide_kernel<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(hp);
    XNS_LAUNCHED(ctx);
  }
  return XNS_OK;
}

int xns_hist_check(xns_ctx *ctx, const HistLaunch &L) {
  unsigned int bad = 0;
  XNS_CUDA(ctx, cudaMemcpyAsync(&bad, L.flags, sizeof(bad), cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (bad) return xns_fail(ctx, XNS_ERR_RANGE, "histogram: " + std::to_string(bad) + " pair distances fall beyond nhist bins");
  return XNS_OK;
}

// The histogram of a set in passes of at most t.max_pairs tile pairs, all adding into d_hist.
static int hist_passes(xns_ctx *ctx, const HistSet &hs, uint32_t nhist, double bin, HistTuning t,
                       unsigned long long *d_hist) {
  if (!t.max_pairs) t.max_pairs = XNS_HIST_PASS_PAIRS;
  int st;
  for (unsigned long long pass = 0;; pass++) {
    t.w_begin = pass * t.max_pairs;
    HistLaunch L;
    if ((st = xns_hist_plan(ctx, hs, nhist, bin, d_hist, t, &L))) return st;
    if (pass == 0 && !t.ordered && L.ntp_total > t.max_pairs) {
      // several passes must form the same tiles: plan again with the cells in input order
      t.ordered = true;
      if ((st = xns_hist_plan(ctx, hs, nhist, bin, d_hist, t, &L))) return st;
    }
    L.zero_hist = pass == 0;
    if (pass == 0 && (st = xns_stage_begin(ctx, STAGE_HIST))) return st;
    if ((st = xns_hist_enqueue(ctx, L))) return st;
    if ((st = xns_hist_check(ctx, L))) return st;
    if (t.w_begin + t.max_pairs >= L.ntp_total) break;
  }
  return xns_stage_end(ctx, STAGE_HIST);
}

int xns_hist_set(xns_ctx *ctx, const HistSet &hs, uint32_t nhist, double bin, unsigned long long *d_hist) {
  return hist_passes(ctx, hs, nhist, bin, HistTuning(), d_hist);
}

int xns_hist_device_shard(xns_ctx *ctx, const DevCoords &dc, uint32_t nhist, double bin, uint32_t shard, uint32_t nshard,
                          unsigned long long *d_hist, unsigned long long max_pairs) {
  HistSet hs;
  hs.x = dc.x;
  hs.y = dc.y;
  hs.z = dc.z;
  hs.el_off = dc.off_el;
  hs.el_n = dc.n_el;
  hs.st.push_back({0, (uint32_t)dc.n_el.size()});
  HistTuning t;
  t.shard = shard;
  t.nshard = nshard;
  t.max_pairs = max_pairs;
  return hist_passes(ctx, hs, nhist, bin, t, d_hist);
}

extern "C" int xns_hist_shard_device(xns_ctx *ctx, const double *xyz_dev, const uint32_t *n_el, uint32_t nel, uint32_t nhist,
                                     double bin, uint32_t shard, uint32_t nshard, uint64_t *hist_dev) {
  if (!ctx) return XNS_ERR_ARG;
  if (!xyz_dev || !hist_dev) return xns_fail(ctx, XNS_ERR_ARG, "hist shard: null device buffer");
  int st;
  DevCoords dc;
  if ((st = xns_timer_start(ctx))) return st;
  if ((st = xns_coords_from_device(ctx, xyz_dev, n_el, nel, &dc))) return st;
  if ((st = xns_hist_device_shard(ctx, dc, nhist, bin, shard, nshard, (unsigned long long *)hist_dev))) return st;
  return xns_timer_stop(ctx);
}

extern "C" int xns_calc_hist_shard(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel,
                                   uint32_t nhist, double bin, uint32_t shard, uint32_t nshard, uint64_t *hist) {
  if (!ctx) return XNS_ERR_ARG;
  if (!hist) return xns_fail(ctx, XNS_ERR_ARG, "hist shard: null output");
  int st;
  DevCoords dc;
  if ((st = xns_upload_coords(ctx, xyz_el, n_el, nel, &dc))) return st;
  void *d_hist;
  size_t bytes = sizeof(unsigned long long) * (size_t)xns_npairs(nel) * nhist;
  if ((st = xns_scratch(ctx, SLOT_HIST, bytes, &d_hist))) return st;
  if ((st = xns_timer_start(ctx))) return st;
  if ((st = xns_hist_device_shard(ctx, dc, nhist, bin, shard, nshard, (unsigned long long *)d_hist))) return st;
  if ((st = xns_timer_stop(ctx))) return st;
  XNS_CUDA(ctx, cudaMemcpyAsync(hist, d_hist, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XNS_OK;
}

int xns_hist_device(xns_ctx *ctx, const DevCoords &dc, uint32_t nhist, double bin, unsigned long long *d_hist) {
  HistSet hs;
  hs.x = dc.x;
  hs.y = dc.y;
  hs.z = dc.z;
  hs.el_off = dc.off_el;
  hs.el_n = dc.n_el;
  hs.st.push_back({0, (uint32_t)dc.n_el.size()});
  return xns_hist_set(ctx, hs, nhist, bin, d_hist);
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

extern "C" int xns_calc_hist_passes(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel,
                                    uint32_t nhist, double bin, uint64_t max_tile_pairs, uint64_t *hist) {
  if (!ctx) return XNS_ERR_ARG;
  if (!hist) return xns_fail(ctx, XNS_ERR_ARG, "hist passes: null output");
  int st;
  DevCoords dc;
  if ((st = xns_upload_coords(ctx, xyz_el, n_el, nel, &dc))) return st;
  void *d_hist;
  size_t bytes = sizeof(unsigned long long) * (size_t)xns_npairs(nel) * nhist;
  if ((st = xns_scratch(ctx, SLOT_HIST, bytes, &d_hist))) return st;
  if ((st = xns_timer_start(ctx))) return st;
  if ((st = xns_hist_device_shard(ctx, dc, nhist, bin, 0, 1, (unsigned long long *)d_hist, max_tile_pairs))) return st;
  if ((st = xns_timer_stop(ctx))) return st;
  XNS_CUDA(ctx, cudaMemcpyAsync(hist, d_hist, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XNS_OK;
}
