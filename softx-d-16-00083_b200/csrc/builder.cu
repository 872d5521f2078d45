// Structure builder: block::calcAtoms (CalcFunctions.cpp:251-392) on the GPU.
//
// The reference builds a block on one host thread:
//   1. every site of the asymmetric unit under every symmetry operation (:268-274);
//   2. for every site, the list of later sites closer than 0.5 A, also across the +-2 neighbouring
//      cells of each replicated axis, each entry with a running occupancy (:275-319): O(sites^2);
//   3. for every copy and unit cell, every site that no earlier site's list claimed draws one uniform
//      number and takes the first list entry whose running occupancy reaches it (:320-385);
//   4. the chosen atom gets the molecule rotation and displacement, the cell and copy transforms, the
//      cut-offs and its own random displacement, and is appended to its element's list.
// Here:
//   (1) one thread per site;
//   (2) a sweep over the triangle of 64 x 64 site tiles, translations culled per tile pair by bounding
//       boxes, exact FP64 distances in the reference's operation order; hits are appended to a buffer,
//       then gathered into per-site lists sorted by site.  Which sites are claimed depends on the lists
//       only, not on the draws, so it is resolved once for all cells by rounds of propagation;
//   (3)+(4) one thread per (copy and cell, unclaimed site): a counting pass, per-CTA offsets, and a
//       writing pass that keeps the reference's order (copy, cell x, y, z, site) within each element.
// All FP64 arithmetic that the reference does with separate multiplies and adds is written with
// __dmul_rn / __dadd_rn so that no contraction into FMA changes a rounding: without random
// displacements the coordinates are bit-identical to the reference's.
//
// Random numbers: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as
// 1, 2, 3", SC 2011), key = the 64-bit seed, counter = (site or symmetry index, copy-and-cell index
// low and high words, block << 8 | purpose).  Two 53-bit uniforms per call.  The reference's
// distributions are kept: occupancy draw U[0,1); displacement direction phi = 2 pi U, theta = pi U;
// radius |N(0, dev)| (Box-Muller here); molecule Euler angles (2 pi U, pi U, 2 pi U).
#include <math.h>

#include <algorithm>
#include <vector>

#include "f32x2.cuh"
#include "xns_internal.cuh"

namespace {

constexpr int MT = 128;         // sites per merge tile (one thread per I row)
constexpr int MAX_T = 125;      // translations: +-2 cells on three axes
constexpr int GEN_THREADS = 256;
constexpr int MAX_NID = 64;

enum Purpose : uint32_t { P_OCC = 0, P_DISP_ANG = 1, P_DISP_RAD = 2, P_MOL_ANG = 3, P_MOL_RAD = 4, P_ROT_A = 5, P_ROT_B = 6 };

struct D3 {
  double x, y, z;
};
__device__ __forceinline__ double m_(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double a_(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double s_(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ D3 add3(D3 a, D3 b) { return D3{a_(a.x, b.x), a_(a.y, b.y), a_(a.z, b.z)}; }
__device__ __forceinline__ D3 sub3(D3 a, D3 b) { return D3{s_(a.x, b.x), s_(a.y, b.y), s_(a.z, b.z)}; }
// vect3d::dot and ::sqr (typedefs.h:128-130): x*t.x + y*t.y + z*t.z, left to right
__device__ __forceinline__ double dot3(D3 a, D3 b) { return a_(a_(m_(a.x, b.x), m_(a.y, b.y)), m_(a.z, b.z)); }
__device__ __forceinline__ double sqr3(D3 a) { return dot3(a, a); }
__device__ __forceinline__ D3 ld3(const double *p) { return D3{p[0], p[1], p[2]}; }
// e[0]*cx + e[1]*cy + e[2]*cz (CalcFunctions.cpp:301, :330)
__device__ __forceinline__ D3 cell_trans(const double *e, double cx, double cy, double cz) {
  return D3{a_(a_(m_(e[0], cx), m_(e[3], cy)), m_(e[6], cz)), a_(a_(m_(e[1], cx), m_(e[4], cy)), m_(e[7], cz)),
            a_(a_(m_(e[2], cx), m_(e[5], cy)), m_(e[8], cz))};
}

struct U4 {
  uint32_t x, y, z, w;
};
__device__ __forceinline__ U4 philox(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
  }
  return c;
}
__device__ __forceinline__ double u53(uint32_t a, uint32_t b) {
  return (double)(((unsigned long long)a << 21) | (b >> 11)) * 0x1.0p-53;
}

struct Rng {
  uint32_t k0, k1, blk;
  __device__ __forceinline__ void draw(uint32_t item, unsigned long long unit, uint32_t purpose, double *u0,
                                       double *u1) const {
    const U4 r = philox(U4{item, (uint32_t)unit, (uint32_t)(unit >> 32), (blk << 8) | purpose}, k0, k1);
    *u0 = u53(r.x, r.y);
    *u1 = u53(r.z, r.w);
  }
  // (R sin(theta) cos(phi), R sin(theta) sin(phi), R cos(theta)) with phi = 2 pi U, theta = pi U and
  // R = |N(0, dev)| (CalcFunctions.cpp:335-340, :366-370)
  __device__ __forceinline__ D3 displacement(uint32_t item, unsigned long long unit, uint32_t p_ang, uint32_t p_rad,
                                             double dev) const {
    double uf, ut, ua, ub;
    draw(item, unit, p_ang, &uf, &ut);
    draw(item, unit, p_rad, &ua, &ub);
    const double fi = m_(2.0 * XNS_PI, uf), theta = m_(XNS_PI, ut);
    const double n = m_(sqrt(m_(-2.0, log(s_(1.0, ua)))), cos(m_(2.0 * XNS_PI, ub)));
    const double R = fabs(m_(dev, n));
    const double st = sin(theta);
    return D3{m_(m_(R, st), cos(fi)), m_(m_(R, st), sin(fi)), m_(R, cos(theta))};
  }
};

// ---- exclusive scan of u32 (three launches), out[n] = total ------------------------------------------

constexpr int SCAN_T = 256, SCAN_PER = 4, SCAN_CHUNK = SCAN_T * SCAN_PER;

__device__ __forceinline__ uint32_t block_exclusive(uint32_t v, uint32_t *warp_tot, uint32_t *total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tot[w] = incl;
  __syncthreads();
  if (w == 0) {
    uint32_t t = lane < nw ? warp_tot[lane] : 0, s = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t u = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += u;
    }
    if (lane < nw) warp_tot[lane] = s - t;
    if (lane == nw - 1) *total = s;
  }
  __syncthreads();
  const uint32_t r = warp_tot[w] + incl - v;
  __syncthreads();
  return r;
}

__global__ void scan_sums_kernel(const uint32_t *in, uint32_t n, uint32_t add, uint32_t *sums) {
  __shared__ uint32_t wt[32], tot;
  const size_t base = (size_t)blockIdx.x * SCAN_CHUNK;
  uint32_t s = 0;
  for (int k = 0; k < SCAN_PER; k++) {
    const size_t i = base + (size_t)k * SCAN_T + threadIdx.x;
    if (i < n) s += in[i] + add;
  }
  block_exclusive(s, wt, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void scan_top_kernel(uint32_t *sums, uint32_t nc, uint32_t *total) {
  __shared__ uint32_t wt[32], tot;
  uint32_t carry = 0;
  for (uint32_t b = 0; b < nc; b += blockDim.x) {
    const uint32_t i = b + threadIdx.x;
    const uint32_t v = i < nc ? sums[i] : 0;
    const uint32_t ex = block_exclusive(v, wt, &tot);
    if (i < nc) sums[i] = carry + ex;
    carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void scan_apply_kernel(const uint32_t *in, uint32_t n, uint32_t add, const uint32_t *sums, uint32_t *out) {
  __shared__ uint32_t wt[32], tot;
  const size_t base = (size_t)blockIdx.x * SCAN_CHUNK + (size_t)threadIdx.x * SCAN_PER;
  uint32_t v[SCAN_PER], s = 0;
  for (int k = 0; k < SCAN_PER; k++) {
    v[k] = base + k < n ? in[base + k] + add : 0;
    s += v[k];
  }
  uint32_t run = sums[blockIdx.x] + block_exclusive(s, wt, &tot);
  for (int k = 0; k < SCAN_PER; k++) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
}

// ---- step 1: sites ------------------------------------------------------------------------------------

struct BlockParams {
  const double *r_atom, *occ, *dev, *p_symm, *r_symm, *r_copy, *cf;  // device copies
  const uint32_t *el_start;                                          // [nid + 1] prefix of natom_el
  uint32_t natom, nid, nsymm, ncopy, ncx, ncy, ncz, S;
  double e[9], r_mean[3], r_mean_c[3], rcut2, rcc2, dev_mol;
  int cutoff, cutoff_copies, ro_mol;
};

// ra0 = pSymm . rAtom (CalcFunctions.cpp:270, :357) and the site position ra0 + rSymm (:271)
__global__ void site_kernel(BlockParams b, double *ax, double *ay, double *az, double *px, double *py, double *pz,
                            uint32_t *type) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= b.S) return;
  const uint32_t ia = s / b.nsymm, is = s % b.nsymm;
  const D3 r = ld3(b.r_atom + 3 * (size_t)ia);
  const double *p = b.p_symm + 9 * (size_t)is;
  const D3 ra0{dot3(ld3(p), r), dot3(ld3(p + 3), r), dot3(ld3(p + 6), r)};
  const D3 pos = add3(ra0, ld3(b.r_symm + 3 * (size_t)is));
  ax[s] = ra0.x, ay[s] = ra0.y, az[s] = ra0.z;
  px[s] = pos.x, py[s] = pos.y, pz[s] = pos.z;
  uint32_t it = 0;
  while (it + 1 < b.nid && ia >= b.el_start[it + 1]) it++;
  type[s] = it;
}

// per tile of MT sites: bounding box lo xyz, hi xyz
__global__ void tile_box_kernel(const double *px, const double *py, const double *pz, uint32_t S, uint32_t ntile,
                                double *box) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntile) return;
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t i = t * MT; i < min(S, (t + 1) * MT); i++) {
    const double v[3] = {px[i], py[i], pz[i]};
    for (int k = 0; k < 3; k++) lo[k] = fmin(lo[k], v[k]), hi[k] = fmax(hi[k], v[k]);
  }
  for (int k = 0; k < 3; k++) box[6 * t + k] = lo[k], box[6 * t + 3 + k] = hi[k];
}

// ---- step 2: pairs of sites closer than 0.5 A -----------------------------------------------------------
//
// FP32 first: each site is stored as float offsets from its tile's box corner, and a tile pair with
// translation t brings tile J's frame into tile I's by delta = oI - oJ + ct (FP64, rounded once).  The
// FP32 squared distance d~^2 = |(a_i + delta) - a_j|^2 then differs from the FP64 one by a bounded
// amount: each component by at most E_k = 2^-23 (2 wI_k + 2 wJ_k + 2 |delta_k| + 1) + 1e-9 (the
// roundings of a_i, a_j, delta and the two subtractions, each at most half an FP32 ulp of a magnitude
// below the bracket, with a factor 2 to spare), so a pair the reference accepts (|d| < 0.5) has
// |d~| < 0.5 + E_x + E_y + E_z and d~^2 below thr = (0.5 + sum E)^2 (1 + 2^-20).  Pairs under thr -- a
// few in a million -- are tested exactly in FP64 with the reference's operations.  Pairs of J rows go
// through the packed f32x2 pipe, four pairs of rows per branch.

struct MergeArgs {
  const double *px, *py, *pz, *box;
  const float *lx, *ly, *lz;  // offsets of each site from its tile's box corner
  double ct[3 * MAX_T];       // translations e0 cx + e1 cy + e2 cz in the reference's loop order
  uint32_t S, ntile, T;
  unsigned long long npairs;  // (I tile, pair of J tiles) pairs: nJ (nJ + 1), nJ = ceil(ntile / 2)
  unsigned long long *hits;
  uint32_t cap;
  uint32_t *nhit, *outdeg, *indeg;
};

__global__ void local_coords_kernel(const double *px, const double *py, const double *pz, const double *box, uint32_t S,
                                    float *lx, float *ly, float *lz) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  const double *b = box + 6 * (s / MT);
  lx[s] = (float)(px[s] - b[0]), ly[s] = (float)(py[s] - b[1]), lz[s] = (float)(pz[s] - b[2]);
}

// exact test of (rAtomCell[i] - rAtomCell[j] + celltrans).sqr() < 0.25 (CalcFunctions.cpp:302)
__device__ __forceinline__ bool exact_hit(const MergeArgs &a, D3 d0, int t) {
  return sqr3(add3(d0, D3{a.ct[3 * t], a.ct[3 * t + 1], a.ct[3 * t + 2]})) < 0.25;
}

// The tile-pair constants of one J half (tile tj, when it exists) for one translation c: whether the
// boxes come within 0.5 A, the frame shift delta = oI - oJ + c and the FP32 threshold (-1 when dead).
struct HalfBox {
  bool live;
  float dx, dy, dz, thr;
};
__device__ __forceinline__ HalfBox half_box(const double *bi, const double *box, unsigned long long tj, uint32_t ntile,
                                            const double *c) {
  HalfBox r{false, 0.f, 0.f, 0.f, -1.f};
  if (tj >= ntile) return r;
  const double *bj = box + 6 * tj;
  double g2 = 0, esum = 0, del[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const double dlo = bi[k] - bj[3 + k] + c[k], dhi = bi[3 + k] - bj[k] + c[k];  // d = ri - rj + c in [dlo, dhi]
    const double g = fmax(0.0, fmax(dlo, -dhi));
    g2 += g * g;
    del[k] = bi[k] - bj[k] + c[k];
    esum += 0x1.0p-23 * (2.0 * (bi[3 + k] - bi[k]) + 2.0 * (bj[3 + k] - bj[k]) + 2.0 * fabs(del[k]) + 1.0) + 1e-9;
  }
  if (!(g2 < 0.25 * (1.0 + 1e-9) + 1e-9)) return r;
  r.live = true;
  r.dx = (float)del[0], r.dy = (float)del[1], r.dz = (float)del[2];
  r.thr = __double2float_ru((0.5 + esum) * (0.5 + esum) * (1.0 + 0x1.0p-20));
  return r;
}

// d~^2 - thr for a pair of J rows, evaluated as one FMA chain: its rounding stays within 2^-21 thr,
// inside the 2^-20 thr of slack in thr, so every pair under the FP32 bound comes out negative
__device__ __forceinline__ xns_f2::f2 merge_excess(xns_f2::f2 xd, xns_f2::f2 yd, xns_f2::f2 zd, xns_f2::f2 nthr,
                                                   xns_f2::f2 xj, xns_f2::f2 yj, xns_f2::f2 zj) {
  using namespace xns_f2;
  const f2 dx = sub(xd, xj), dy = sub(yd, yj), dz = sub(zd, zj);
  return fma(dz, dz, fma(dy, dy, fma(dx, dx, nthr)));
}

// A CTA takes an I tile (MT sites, one per thread) against a J tile of 2 MT sites (two consecutive
// tiles, each in its own frame): tile pair p of the triangle ti <= 2 tj2 + 1 decodes as
// tj2 (tj2 + 1) <= p < (tj2 + 1)(tj2 + 2), ti = p - tj2 (tj2 + 1).
__global__ void __launch_bounds__(128) merge_kernel(const __grid_constant__ MergeArgs a) {
  using namespace xns_f2;
  __shared__ f2 jx2[MT], jy2[MT], jz2[MT];  // the J tile's 2 MT sites as MT pairs
  __shared__ float sdel[MAX_T][2][4];       // per live translation and J half: delta x y z, thr (< 0: dead)
  __shared__ uint8_t alive[MAX_T];
  __shared__ int nalive;
  for (unsigned long long p = blockIdx.x; p < a.npairs; p += gridDim.x) {
    unsigned long long tj2 = (unsigned long long)((sqrt(4.0 * (double)p + 1.0) - 1.0) * 0.5);
    while (tj2 * (tj2 + 1) > p) tj2--;
    while ((tj2 + 1) * (tj2 + 2) <= p) tj2++;
    const unsigned long long ti = p - tj2 * (tj2 + 1);
    if (ti >= a.ntile) continue;  // uniform across the CTA: an odd tile count leaves no I tile here
    __syncthreads();
    if (threadIdx.x == 0) nalive = 0;
    __syncthreads();
    // a translation can only give a hit when the boxes come closer than 0.5 A (with slack for rounding);
    // live translations (live for either half) are kept in loop order, so the first one that hits a
    // pair is found first
    const double *bi = a.box + 6 * ti;
    if (threadIdx.x < 32) {
      for (uint32_t t0 = 0; t0 < a.T; t0 += 32) {
        const uint32_t t = t0 + threadIdx.x;
        const HalfBox h0 = t < a.T ? half_box(bi, a.box, 2 * tj2, a.ntile, a.ct + 3 * t) : HalfBox{false, 0.f, 0.f, 0.f, -1.f};
        const HalfBox h1 = t < a.T ? half_box(bi, a.box, 2 * tj2 + 1, a.ntile, a.ct + 3 * t) : HalfBox{false, 0.f, 0.f, 0.f, -1.f};
        const bool live = h0.live || h1.live;
        const uint32_t m = __ballot_sync(0xffffffffu, live);
        if (live) {
          const int slot = nalive + __popc(m & ((1u << threadIdx.x) - 1));
          alive[slot] = (uint8_t)t;
          sdel[slot][0][0] = h0.dx, sdel[slot][0][1] = h0.dy, sdel[slot][0][2] = h0.dz, sdel[slot][0][3] = h0.thr;
          sdel[slot][1][0] = h1.dx, sdel[slot][1][1] = h1.dy, sdel[slot][1][2] = h1.dz, sdel[slot][1][3] = h1.thr;
        }
        __syncwarp();
        if (threadIdx.x == 0) nalive += __popc(m);
        __syncwarp();
      }
    }
    {
      const size_t j = tj2 * 2 * MT + 2 * threadIdx.x;
      // rows past the end sit far away and never pass the FP32 test
      const float x0 = j < a.S ? a.lx[j] : 1e30f, y0 = j < a.S ? a.ly[j] : 1e30f, z0 = j < a.S ? a.lz[j] : 1e30f;
      const float x1 = j + 1 < a.S ? a.lx[j + 1] : 1e30f, y1 = j + 1 < a.S ? a.ly[j + 1] : 1e30f,
                  z1 = j + 1 < a.S ? a.lz[j + 1] : 1e30f;
      jx2[threadIdx.x] = pack(x0, x1), jy2[threadIdx.x] = pack(y0, y1), jz2[threadIdx.x] = pack(z0, z1);
    }
    __syncthreads();
    const int na = nalive;
    if (na == 0) continue;
    const uint32_t i = (uint32_t)(ti * MT) + threadIdx.x;
    if (i >= a.S) continue;
    const float xi = a.lx[i], yi = a.ly[i], zi = a.lz[i];
    // the first half holds only sites below every i of the I tile when the I tile is the second tile
    const int h0 = ti == 2 * tj2 + 1 ? 1 : 0;
    for (int s = 0; s < na; s++) {
      for (int h = h0; h < 2; h++) {
        const float thr = sdel[s][h][3];
        if (thr < 0.f) continue;
        const f2 xd = splat(xi + sdel[s][h][0]), yd = splat(yi + sdel[s][h][1]), zd = splat(zi + sdel[s][h][2]);
        const f2 nthr = splat(-thr);
        for (int k0 = h * (MT / 2); k0 < (h + 1) * (MT / 2); k0 += 4) {
          unsigned long long any = 0;  // sign bits of four pairs of J rows
#pragma unroll
          for (int u = 0; u < 4; u++) any |= merge_excess(xd, yd, zd, nthr, jx2[k0 + u], jy2[k0 + u], jz2[k0 + u]);
          if (!(any & 0x8000000080000000ull)) continue;
          for (int u = 0; u < 4; u++) {
            const unsigned long long e2 = merge_excess(xd, yd, zd, nthr, jx2[k0 + u], jy2[k0 + u], jz2[k0 + u]);
            for (int hh = 0; hh < 2; hh++) {
              const uint32_t j = (uint32_t)(tj2 * 2 * MT) + 2 * (k0 + u) + hh;
              if (!((e2 >> (32 * hh + 31)) & 1) || j <= i || j >= a.S) continue;
              const D3 d0 = sub3(D3{a.px[i], a.py[i], a.pz[i]}, D3{a.px[j], a.py[j], a.pz[j]});
              // record the pair once: at the first live translation that hits it
              if (!exact_hit(a, d0, alive[s])) continue;
              bool earlier = false;
              for (int e = 0; e < s && !earlier; e++) earlier = exact_hit(a, d0, alive[e]);
              if (earlier) continue;
              const uint32_t pos = atomicAdd(a.nhit, 1u);
              if (pos < a.cap) a.hits[pos] = ((unsigned long long)i << 32) | j;
              atomicAdd(a.outdeg + i, 1u);
              atomicAdd(a.indeg + j, 1u);
            }
          }
        }
      }
    }
  }
}

// list of site i: i itself, then the later sites it hits (CalcFunctions.cpp:283-287, :303-308)
__global__ void list_self_kernel(const uint32_t *off, uint32_t S, uint32_t *list) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < S) list[off[i]] = i;
}
__global__ void list_scatter_kernel(const unsigned long long *hits, uint32_t nhit, const uint32_t *off,
                                    uint32_t *cursor, uint32_t *list) {
  const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= nhit) return;
  const uint32_t i = (uint32_t)(hits[h] >> 32), j = (uint32_t)hits[h];
  list[off[i] + 1 + atomicAdd(cursor + i, 1u)] = j;
}
// sort each list by site (the reference appends in increasing j), then the running occupancy:
// the previous entry's, plus the entry's own when its element differs from the previous entry's
// (CalcFunctions.cpp:305-306)
__global__ void list_finish_kernel(const uint32_t *off, uint32_t S, uint32_t nsymm, const uint32_t *type,
                                   const double *occ, uint32_t *list, double *cum) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S) return;
  const uint32_t b = off[i], e = off[i + 1];
  for (uint32_t m = b + 2; m < e; m++) {
    const uint32_t v = list[m];
    uint32_t k = m;
    while (k > b + 1 && list[k - 1] > v) list[k] = list[k - 1], k--;
    list[k] = v;
  }
  double c = occ[i / nsymm];
  uint32_t prev = type[i];
  cum[b] = c;
  for (uint32_t m = b + 1; m < e; m++) {
    const uint32_t j = list[m];
    if (type[j] != prev) c += occ[j / nsymm];
    prev = type[j];
    cum[m] = c;
  }
}

// ---- which sites draw: a site draws unless an earlier drawing site lists it (CalcFunctions.cpp:349-351)
// state: 0 open, 1 draws, 2 claimed.  A site with no earlier site listing it draws; a site listed by a
// drawing site is claimed; a site all of whose listers are claimed draws.
__global__ void claim_init_kernel(const uint32_t *indeg, uint32_t S, uint8_t *state, uint8_t *done,
                                  uint32_t *folcnt) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S) return;
  state[i] = indeg[i] == 0 ? 1 : 0;
  done[i] = 0;
  folcnt[i] = 0;
}
__global__ void claim_propagate_kernel(const uint32_t *off, const uint32_t *list, uint32_t S, uint8_t *state,
                                       uint8_t *done, uint32_t *folcnt) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S || done[i]) return;
  const uint8_t st = ((volatile uint8_t *)state)[i];
  if (st == 0) return;
  done[i] = 1;
  for (uint32_t m = off[i] + 1; m < off[i + 1]; m++) {
    if (st == 1)
      ((volatile uint8_t *)state)[list[m]] = 2;
    else
      atomicAdd(folcnt + list[m], 1u);
  }
}
__global__ void claim_resolve_kernel(const uint32_t *indeg, const uint32_t *folcnt, uint32_t S, uint8_t *state,
                                     uint32_t *open) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S || state[i] != 0) return;
  if (folcnt[i] == indeg[i])
    state[i] = 1;
  else
    atomicAdd(open, 1u);
}
// the reference's own sequential rule, for chains that the rounds would resolve too slowly
__global__ void claim_sequential_kernel(const uint32_t *off, const uint32_t *list, uint32_t S, uint8_t *state) {
  if (threadIdx.x || blockIdx.x) return;
  for (uint32_t i = 0; i < S; i++) state[i] = 0;
  for (uint32_t i = 0; i < S; i++) {
    if (state[i] == 2) continue;
    state[i] = 1;
    for (uint32_t m = off[i] + 1; m < off[i + 1]; m++) state[list[m]] = 2;
  }
}
__global__ void claim_flags_kernel(const uint8_t *state, uint32_t S, uint32_t *flag) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < S) flag[i] = state[i] == 1;
}
__global__ void leaders_kernel(const uint32_t *flag, const uint32_t *pos, uint32_t S, uint32_t *lead) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < S && flag[i]) lead[pos[i]] = i;
}

// ---- steps 3 and 4: the atoms -------------------------------------------------------------------------

struct GenArgs {
  BlockParams b;
  const double *ax, *ay, *az;  // ra0 per site
  const uint32_t *type, *off, *list, *lead;
  const double *cum;
  uint32_t nlead;
  unsigned long long items, per_cta;
  Rng rng;
};

// One (copy and cell, drawing site) item: the block-local element of the atom it places, or -1.
__device__ int gen_atom(const GenArgs &g, unsigned long long item, D3 *out) {
  const BlockParams &b = g.b;
  const unsigned long long unit = item / g.nlead;
  const uint32_t s = g.lead[item - unit * g.nlead];
  unsigned long long t = unit;
  const uint32_t cz = (uint32_t)(t % b.ncz);
  t /= b.ncz;
  const uint32_t cy = (uint32_t)(t % b.ncy);
  t /= b.ncy;
  const uint32_t cx = (uint32_t)(t % b.ncx);
  const uint32_t copy = (uint32_t)(t / b.ncx);
  double randval, unused;
  g.rng.draw(s, unit, P_OCC, &randval, &unused);
  uint32_t chosen = 0xffffffffu;
  for (uint32_t m = g.off[s]; m < g.off[s + 1]; m++)
    if (randval <= g.cum[m]) {
      chosen = g.list[m];
      break;
    }
  if (chosen == 0xffffffffu) return -1;
  const uint32_t ia = chosen / b.nsymm, is = chosen % b.nsymm;
  D3 ra1{g.ax[chosen], g.ay[chosen], g.az[chosen]};
  if (b.ro_mol) {  // CalcFunctions.cpp:341-347, :358
    double u0, u1, u2, u3;
    g.rng.draw(is, unit, P_ROT_A, &u0, &u1);
    g.rng.draw(is, unit, P_ROT_B, &u2, &u3);
    const double ex = m_(2.0 * XNS_PI, u0), ey = m_(XNS_PI, u1), ez = m_(2.0 * XNS_PI, u2);
    const double cx_ = cos(ex), cy_ = cos(ey), cz_ = cos(ez), sx = sin(ex), sy = sin(ey), sz = sin(ez);
    const D3 r0{s_(m_(cx_, cy_), m_(m_(sx, sy), cz_)), s_(m_(-cx_, sy), m_(m_(sx, cz_), cy_)), m_(sx, sz)};
    const D3 r1{a_(m_(sx, cy_), m_(m_(cx_, sy), cz_)), a_(m_(-sx, sy), m_(m_(cx_, cy_), cz_)), m_(-cx_, sz)};
    const D3 r2{m_(sz, sy), m_(sz, cy_), cz_};
    ra1 = D3{dot3(ra1, r0), dot3(ra1, r1), dot3(ra1, r2)};
  }
  D3 rmd{0.0, 0.0, 0.0};
  if (b.dev_mol >= 1.e-7) rmd = g.rng.displacement(is, unit, P_MOL_ANG, P_MOL_RAD, b.dev_mol);  // :332-340
  const D3 ct = cell_trans(b.e, (double)cx, (double)cy, (double)cz);
  ra1 = add3(ra1, add3(add3(ld3(b.r_symm + 3 * (size_t)is), ct), rmd));  // :360
  const D3 rm = ld3(b.r_mean);
  if (b.cutoff && !(sqr3(sub3(ra1, rm)) <= b.rcut2)) return -1;  // :361
  const D3 d = sub3(ra1, rm);
  const double *cf = b.cf + 9 * (size_t)copy;
  ra1 = add3(ld3(b.r_copy + 3 * (size_t)copy), D3{dot3(d, ld3(cf)), dot3(d, ld3(cf + 3)), dot3(d, ld3(cf + 6))});
  const double dv = b.dev[ia];
  if (dv >= 1.e-7) ra1 = add3(ra1, g.rng.displacement(s, unit, P_DISP_ANG, P_DISP_RAD, dv));  // :364-371
  if (b.cutoff_copies && !(sqr3(sub3(ra1, ld3(b.r_mean_c))) <= b.rcc2)) return -1;  // :372
  *out = ra1;
  return (int)g.type[chosen];
}

__global__ void __launch_bounds__(GEN_THREADS) gen_count_kernel(const __grid_constant__ GenArgs g, uint32_t *cta_cnt) {
  __shared__ uint32_t cnt[MAX_NID];
  for (int k = threadIdx.x; k < MAX_NID; k += blockDim.x) cnt[k] = 0;
  __syncthreads();
  const unsigned long long lo = blockIdx.x * g.per_cta, hi = min(g.items, lo + g.per_cta);
  for (unsigned long long it = lo + threadIdx.x; it < hi; it += GEN_THREADS) {
    D3 r;
    const int e = gen_atom(g, it, &r);
    if (e >= 0) atomicAdd(cnt + e, 1u);
  }
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < g.b.nid; k += blockDim.x) cta_cnt[(size_t)blockIdx.x * g.b.nid + k] = cnt[k];
}

// per element (one warp each): exclusive offsets of the CTAs' counts and the block's total
__global__ void gen_offsets_kernel(uint32_t *cta_cnt, uint32_t ncta, uint32_t nid, uint32_t *total) {
  const uint32_t k = blockIdx.x, lane = threadIdx.x;
  uint32_t run = 0;
  for (uint32_t c0 = 0; c0 < ncta; c0 += 32) {
    const uint32_t c = c0 + lane;
    const uint32_t v = c < ncta ? cta_cnt[(size_t)c * nid + k] : 0;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (c < ncta) cta_cnt[(size_t)c * nid + k] = run + incl - v;
    run += __shfl_sync(0xffffffffu, incl, 31);
  }
  if (lane == 0) total[k] = run;
}

// dst[k]: first atom slot of block element k in the output
__global__ void __launch_bounds__(GEN_THREADS) gen_write_kernel(const __grid_constant__ GenArgs g, const uint32_t *cta_off,
                                                                 const unsigned long long *dst, double *out) {
  constexpr int NW = GEN_THREADS / 32;
  __shared__ uint32_t wcnt[NW][MAX_NID], cur[MAX_NID];
  const uint32_t nid = g.b.nid;
  for (uint32_t k = threadIdx.x; k < MAX_NID; k += blockDim.x) {
    cur[k] = k < nid ? cta_off[(size_t)blockIdx.x * nid + k] : 0;
    for (int w = 0; w < NW; w++) wcnt[w][k] = 0;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned long long lo = blockIdx.x * g.per_cta, hi = min(g.items, lo + g.per_cta);
  for (unsigned long long base = lo; base < hi; base += GEN_THREADS) {
    const unsigned long long it = base + threadIdx.x;
    D3 r;
    const int e = it < hi ? gen_atom(g, it, &r) : -1;
    const uint32_t peers = __match_any_sync(0xffffffffu, e);
    const uint32_t rank = __popc(peers & ((1u << lane) - 1));
    if (e >= 0 && rank == 0) wcnt[warp][e] = __popc(peers);
    __syncthreads();
    if (e >= 0) {
      uint32_t o = cur[e] + rank;
      for (int w = 0; w < warp; w++) o += wcnt[w][e];
      double *p = out + 3 * (dst[e] + o);
      p[0] = r.x, p[1] = r.y, p[2] = r.z;
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < nid; k += blockDim.x) {
      uint32_t s = 0;
      for (int w = 0; w < NW; w++) s += wcnt[w][k], wcnt[w][k] = 0;
      cur[k] += s;
    }
    __syncthreads();
  }
}

// ---- host ------------------------------------------------------------------------------------------------

unsigned blocks_for(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

// Device allocations of one call, freed in order on the stream when the call ends.
struct Arena {
  xns_ctx *ctx;
  std::vector<void *> ptrs;
  explicit Arena(xns_ctx *c) : ctx(c) {}
  ~Arena() {
    for (void *p : ptrs) cudaFreeAsync(p, ctx->stream);
  }
  template <class T>
  int get(size_t n, T **out) {
    void *p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, std::max<size_t>(n * sizeof(T), 16), ctx->stream);
    if (e != cudaSuccess) return xns_cuda_fail(ctx, e, "cudaMallocAsync");
    ptrs.push_back(p);
    *out = (T *)p;
    return XNS_OK;
  }
};

#define XNS_TRY(x)              \
  do {                          \
    int _s = (x);               \
    if (_s != XNS_OK) return _s; \
  } while (0)

int scan_u32(xns_ctx *ctx, Arena &ar, const uint32_t *in, uint32_t n, uint32_t add, uint32_t *out, uint32_t *total) {
  const uint32_t nc = std::max(1u, (uint32_t)((n + SCAN_CHUNK - 1) / SCAN_CHUNK));
  uint32_t *sums;
  XNS_TRY(ar.get(nc, &sums));
  scan_sums_kernel<<<nc, SCAN_T, 0, ctx->stream>>>(in, n, add, sums);
  XNS_LAUNCHED(ctx);
  scan_top_kernel<<<1, 1024, 0, ctx->stream>>>(sums, nc, out + n);
  XNS_LAUNCHED(ctx);
  scan_apply_kernel<<<nc, SCAN_T, 0, ctx->stream>>>(in, n, add, sums, out);
  XNS_LAUNCHED(ctx);
  if (total) XNS_CUDA(ctx, cudaMemcpyAsync(total, out + n, 4, cudaMemcpyDeviceToHost, ctx->stream));
  return XNS_OK;
}

// State of one block between the counting and the writing pass.
struct BlockRun {
  GenArgs g{};
  uint32_t ncta = 0;
  uint32_t *cta_cnt = nullptr;
  std::vector<uint32_t> total;  // atoms per block element
};

int check_block(xns_ctx *ctx, const xns_block &bk, uint32_t nel) {
  if (bk.natom == 0) return XNS_OK;
  if (!bk.natom_el || !bk.id || !bk.r_atom || !bk.occ || !bk.dev || !bk.p_symm || !bk.r_symm || !bk.r_copy || !bk.cf)
    return xns_fail(ctx, XNS_ERR_ARG, "xns_build_atoms: a block array is NULL");
  if (bk.nid == 0 || bk.nid > MAX_NID || bk.nsymm == 0 || bk.ncopy == 0 || !bk.ncell[0] || !bk.ncell[1] || !bk.ncell[2])
    return xns_fail(ctx, XNS_ERR_ARG, "xns_build_atoms: nid must be 1..64 and nsymm, ncopy, ncell >= 1");
  if ((uint64_t)bk.natom * bk.nsymm >= (1ull << 31))
    return xns_fail(ctx, XNS_ERR_ARG, "xns_build_atoms: natom * nsymm must stay below 2^31");
  uint64_t s = 0;
  for (uint32_t k = 0; k < bk.nid; k++) {
    if (bk.id[k] >= nel) return xns_fail(ctx, XNS_ERR_ARG, "xns_build_atoms: block element id >= nel");
    s += bk.natom_el[k];
  }
  if (s != bk.natom) return xns_fail(ctx, XNS_ERR_ARG, "xns_build_atoms: natom_el does not sum to natom");
  return XNS_OK;
}

// Steps 1-3 and the counting pass of one block.
int plan_block(xns_ctx *ctx, Arena &ar, const xns_block &bk, uint32_t blk, uint64_t seed, BlockRun *run) {
  cudaStream_t st = ctx->stream;
  const uint32_t S = bk.natom * bk.nsymm;
  BlockParams &b = run->g.b;
  b.natom = bk.natom, b.nid = bk.nid, b.nsymm = bk.nsymm, b.ncopy = bk.ncopy;
  b.ncx = bk.ncell[0], b.ncy = bk.ncell[1], b.ncz = bk.ncell[2], b.S = S;
  for (int k = 0; k < 9; k++) b.e[k] = bk.e[k / 3][k % 3];
  for (int k = 0; k < 3; k++) b.r_mean[k] = bk.r_mean[k];
  // rMeanC: the mean copy position (CalcFunctions.cpp:264-267)
  double mc[3] = {0, 0, 0};
  for (uint32_t c = 0; c < bk.ncopy; c++)
    for (int k = 0; k < 3; k++) mc[k] += bk.r_copy[3 * c + k];
  for (int k = 0; k < 3; k++) b.r_mean_c[k] = mc[k] / (double)bk.ncopy;
  b.rcut2 = bk.rcut * bk.rcut;
  b.rcc2 = bk.rcut_copies * bk.rcut_copies;
  b.dev_mol = bk.dev_mol;
  b.cutoff = bk.cutoff, b.cutoff_copies = bk.cutoff_copies, b.ro_mol = bk.ro_mol;

  // block arrays: one upload
  std::vector<double> hd;
  auto put = [&](const double *p, size_t n) {
    size_t o = hd.size();
    hd.insert(hd.end(), p, p + n);
    return o;
  };
  const size_t o_ra = put(bk.r_atom, 3 * (size_t)bk.natom), o_occ = put(bk.occ, bk.natom), o_dev = put(bk.dev, bk.natom),
               o_ps = put(bk.p_symm, 9 * (size_t)bk.nsymm), o_rs = put(bk.r_symm, 3 * (size_t)bk.nsymm),
               o_rc = put(bk.r_copy, 3 * (size_t)bk.ncopy), o_cf = put(bk.cf, 9 * (size_t)bk.ncopy);
  std::vector<uint32_t> el_start(bk.nid + 1, 0);
  for (uint32_t k = 0; k < bk.nid; k++) el_start[k + 1] = el_start[k] + bk.natom_el[k];
  double *dd;
  uint32_t *d_el;
  XNS_TRY(ar.get(hd.size(), &dd));
  XNS_TRY(ar.get(el_start.size(), &d_el));
  XNS_CUDA(ctx, cudaMemcpyAsync(dd, hd.data(), hd.size() * 8, cudaMemcpyHostToDevice, st));
  XNS_CUDA(ctx, cudaMemcpyAsync(d_el, el_start.data(), el_start.size() * 4, cudaMemcpyHostToDevice, st));
  b.r_atom = dd + o_ra, b.occ = dd + o_occ, b.dev = dd + o_dev, b.p_symm = dd + o_ps, b.r_symm = dd + o_rs;
  b.r_copy = dd + o_rc, b.cf = dd + o_cf, b.el_start = d_el;

  // step 1
  double *site;
  uint32_t *type;
  XNS_TRY(ar.get(6 * (size_t)S, &site));
  XNS_TRY(ar.get(S, &type));
  double *ax = site, *ay = site + S, *az = site + 2 * (size_t)S, *px = site + 3 * (size_t)S, *py = site + 4 * (size_t)S,
         *pz = site + 5 * (size_t)S;
  site_kernel<<<blocks_for(S, 256), 256, 0, st>>>(b, ax, ay, az, px, py, pz, type);
  XNS_LAUNCHED(ctx);

  // step 2
  MergeArgs ma{};
  int T = 0;
  {
    int st_[3], fin[3];
    for (int k = 0; k < 3; k++) {
      st_[k] = bk.ncell[k] == 1 ? 0 : -2;
      fin[k] = bk.ncell[k] == 1 ? 1 : 3;
    }
    // the translations are formed on the host in the reference's operation order: plain double
    // multiplies and adds, no fused multiply-add on the host compiler's x86-64 target
    for (int cx = st_[0]; cx < fin[0]; cx++)
      for (int cy = st_[1]; cy < fin[1]; cy++)
        for (int cz = st_[2]; cz < fin[2]; cz++, T++)
          for (int k = 0; k < 3; k++) {
            volatile double p0 = bk.e[0][k] * (double)cx, p1 = bk.e[1][k] * (double)cy, p2 = bk.e[2][k] * (double)cz;
            volatile double s01 = p0 + p1;
            ma.ct[3 * T + k] = s01 + p2;
          }
  }
  const uint32_t ntile = (S + MT - 1) / MT;
  double *box;
  XNS_TRY(ar.get(6 * (size_t)ntile, &box));
  tile_box_kernel<<<blocks_for(ntile, 128), 128, 0, st>>>(px, py, pz, S, ntile, box);
  XNS_LAUNCHED(ctx);
  float *loc;
  XNS_TRY(ar.get(3 * (size_t)S, &loc));
  local_coords_kernel<<<blocks_for(S, 256), 256, 0, st>>>(px, py, pz, box, S, loc, loc + S, loc + 2 * (size_t)S);
  XNS_LAUNCHED(ctx);
  ma.lx = loc, ma.ly = loc + S, ma.lz = loc + 2 * (size_t)S;
  uint32_t *deg, *nhit;
  XNS_TRY(ar.get(2 * (size_t)S + 1, &deg));
  uint32_t *outdeg = deg, *indeg = deg + S;
  nhit = deg + 2 * (size_t)S;
  ma.px = px, ma.py = py, ma.pz = pz, ma.box = box, ma.S = S, ma.ntile = ntile, ma.T = (uint32_t)T;
  const unsigned long long nj2 = (ntile + 1) / 2;
  ma.npairs = nj2 * (nj2 + 1);
  ma.outdeg = outdeg, ma.indeg = indeg, ma.nhit = nhit;
  uint32_t cap = std::max<uint32_t>(S, 1u << 16), h_nhit = 0;
  for (int attempt = 0; attempt < 2; attempt++) {
    unsigned long long *hits;
    XNS_TRY(ar.get(cap, &hits));
    ma.hits = hits, ma.cap = cap;
    XNS_CUDA(ctx, cudaMemsetAsync(deg, 0, (2 * (size_t)S + 1) * 4, st));
    const unsigned grid = (unsigned)std::min<unsigned long long>(ma.npairs, (unsigned long long)ctx->num_sms * 16);
    XNS_TRY(xns_stage_begin(ctx, STAGE_MERGE));
    merge_kernel<<<grid, 128, 0, st>>>(ma);
    XNS_LAUNCHED(ctx);
    XNS_TRY(xns_stage_end(ctx, STAGE_MERGE));
    XNS_CUDA(ctx, cudaMemcpyAsync(&h_nhit, nhit, 4, cudaMemcpyDeviceToHost, st));
    XNS_CUDA(ctx, cudaStreamSynchronize(st));
    if (h_nhit <= cap) break;
    if (attempt == 1 || h_nhit > (1u << 30)) return xns_fail(ctx, XNS_ERR_ARG, "xns_build_atoms: too many overlapping sites");
    cap = h_nhit;
  }
  uint32_t *off, *list, *cursor, L = 0;
  XNS_TRY(ar.get((size_t)S + 1, &off));
  XNS_TRY(scan_u32(ctx, ar, outdeg, S, 1, off, nullptr));
  L = S + h_nhit;
  double *cum;
  XNS_TRY(ar.get(L, &list));
  XNS_TRY(ar.get(L, &cum));
  XNS_TRY(ar.get(S, &cursor));
  XNS_CUDA(ctx, cudaMemsetAsync(cursor, 0, (size_t)S * 4, st));
  list_self_kernel<<<blocks_for(S, 256), 256, 0, st>>>(off, S, list);
  XNS_LAUNCHED(ctx);
  if (h_nhit) {
    list_scatter_kernel<<<blocks_for(h_nhit, 256), 256, 0, st>>>(ma.hits, h_nhit, off, cursor, list);
    XNS_LAUNCHED(ctx);
  }
  list_finish_kernel<<<blocks_for(S, 128), 128, 0, st>>>(off, S, bk.nsymm, type, b.occ, list, cum);
  XNS_LAUNCHED(ctx);

  // which sites draw
  uint8_t *state, *done;
  uint32_t *folcnt, *open;
  XNS_TRY(ar.get(2 * (size_t)S, &state));
  done = state + S;
  XNS_TRY(ar.get((size_t)S + 1, &folcnt));
  open = folcnt + S;
  claim_init_kernel<<<blocks_for(S, 256), 256, 0, st>>>(indeg, S, state, done, folcnt);
  XNS_LAUNCHED(ctx);
  if (h_nhit) {
    uint32_t h_open = 1;
    for (int round = 0; round < 64 && h_open; round++) {
      XNS_CUDA(ctx, cudaMemsetAsync(open, 0, 4, st));
      claim_propagate_kernel<<<blocks_for(S, 256), 256, 0, st>>>(off, list, S, state, done, folcnt);
      XNS_LAUNCHED(ctx);
      claim_resolve_kernel<<<blocks_for(S, 256), 256, 0, st>>>(indeg, folcnt, S, state, open);
      XNS_LAUNCHED(ctx);
      XNS_CUDA(ctx, cudaMemcpyAsync(&h_open, open, 4, cudaMemcpyDeviceToHost, st));
      XNS_CUDA(ctx, cudaStreamSynchronize(st));
    }
    if (h_open) {
      claim_sequential_kernel<<<1, 1, 0, st>>>(off, list, S, state);
      XNS_LAUNCHED(ctx);
    }
  }
  uint32_t *flag, *pos, *lead, nlead = 0;
  XNS_TRY(ar.get(S, &flag));
  XNS_TRY(ar.get((size_t)S + 1, &pos));
  XNS_TRY(ar.get(S, &lead));
  claim_flags_kernel<<<blocks_for(S, 256), 256, 0, st>>>(state, S, flag);
  XNS_LAUNCHED(ctx);
  XNS_TRY(scan_u32(ctx, ar, flag, S, 0, pos, &nlead));
  leaders_kernel<<<blocks_for(S, 256), 256, 0, st>>>(flag, pos, S, lead);
  XNS_LAUNCHED(ctx);
  XNS_CUDA(ctx, cudaStreamSynchronize(st));

  // counting pass
  GenArgs &g = run->g;
  g.ax = ax, g.ay = ay, g.az = az, g.type = type, g.off = off, g.list = list, g.lead = lead, g.cum = cum;
  g.nlead = nlead;
  g.rng = Rng{(uint32_t)seed, (uint32_t)(seed >> 32), blk};
  const unsigned long long units = (unsigned long long)bk.ncopy * bk.ncell[0] * bk.ncell[1] * bk.ncell[2];
  g.items = units * nlead;
  run->total.assign(bk.nid, 0);
  if (g.items == 0) return XNS_OK;
  const unsigned long long max_cta = (unsigned long long)ctx->num_sms * 8;
  unsigned long long per = (g.items + max_cta - 1) / max_cta;
  per = (per + GEN_THREADS - 1) / GEN_THREADS * GEN_THREADS;
  g.per_cta = per;
  run->ncta = (uint32_t)((g.items + per - 1) / per);
  uint32_t *tot;
  XNS_TRY(ar.get((size_t)run->ncta * bk.nid, &run->cta_cnt));
  XNS_TRY(ar.get(bk.nid, &tot));
  gen_count_kernel<<<run->ncta, GEN_THREADS, 0, st>>>(g, run->cta_cnt);
  XNS_LAUNCHED(ctx);
  gen_offsets_kernel<<<bk.nid, 32, 0, st>>>(run->cta_cnt, run->ncta, bk.nid, tot);
  XNS_LAUNCHED(ctx);
  XNS_CUDA(ctx, cudaMemcpyAsync(run->total.data(), tot, 4 * (size_t)bk.nid, cudaMemcpyDeviceToHost, st));
  XNS_CUDA(ctx, cudaStreamSynchronize(st));
  return XNS_OK;
}

}  // namespace

extern "C" int xns_build_atoms(xns_ctx *ctx, const xns_block *blocks, uint32_t nblocks, uint32_t nel, uint64_t seed,
                               uint32_t *n_el, uint32_t *n_all, const double **xyz_dev) {
  if (!ctx) return XNS_ERR_ARG;
  if (!blocks || !n_el || !xyz_dev || nel == 0 || nel > MAX_NID)
    return xns_fail(ctx, XNS_ERR_ARG, "xns_build_atoms: blocks, n_el and xyz_dev are required and nel must be 1..64");
  for (uint32_t ib = 0; ib < nblocks; ib++) XNS_TRY(check_block(ctx, blocks[ib], nel));
  XNS_TRY(xns_timer_start(ctx));
  Arena ar(ctx);
  std::vector<BlockRun> runs(nblocks);
  for (uint32_t ib = 0; ib < nblocks; ib++)
    if (blocks[ib].natom) XNS_TRY(plan_block(ctx, ar, blocks[ib], ib, seed, &runs[ib]));
  // element-major output: element g holds block 0's atoms of g, then block 1's, ...
  std::vector<unsigned long long> count(nel, 0), start(nel + 1, 0);
  for (uint32_t ib = 0; ib < nblocks; ib++)
    for (uint32_t k = 0; k < runs[ib].total.size(); k++) count[blocks[ib].id[k]] += runs[ib].total[k];
  for (uint32_t e = 0; e < nel; e++) start[e + 1] = start[e] + count[e];
  if (start[nel] >= 0xffffffffull) return xns_fail(ctx, XNS_ERR_ARG, "xns_build_atoms: 2^32 - 1 atoms or more");
  void *outv;
  XNS_TRY(xns_scratch(ctx, SLOT_ATOMS, 24 * (size_t)std::max<unsigned long long>(start[nel], 1), &outv));
  double *out = (double *)outv;
  std::vector<unsigned long long> filled(nel, 0);
  uint32_t o_all = 0;
  for (uint32_t ib = 0; ib < nblocks; ib++) {
    const xns_block &bk = blocks[ib];
    BlockRun &r = runs[ib];
    if (bk.natom && r.g.items) {
      std::vector<unsigned long long> dst(bk.nid);
      for (uint32_t k = 0; k < bk.nid; k++) dst[k] = start[bk.id[k]] + filled[bk.id[k]];
      unsigned long long *d_dst;
      XNS_TRY(ar.get(bk.nid, &d_dst));
      XNS_CUDA(ctx, cudaMemcpyAsync(d_dst, dst.data(), 8 * (size_t)bk.nid, cudaMemcpyHostToDevice, ctx->stream));
      XNS_TRY(xns_stage_begin(ctx, STAGE_FILL));
      gen_write_kernel<<<r.ncta, GEN_THREADS, 0, ctx->stream>>>(r.g, r.cta_cnt, d_dst, out);
      XNS_LAUNCHED(ctx);
      XNS_TRY(xns_stage_end(ctx, STAGE_FILL));
      XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // dst lives on this host frame
    }
    for (uint32_t k = 0; k < bk.nid; k++) {
      const uint32_t c = k < r.total.size() ? r.total[k] : 0;
      if (c) filled[bk.id[k]] += c;
      if (n_all) n_all[o_all + k] = c;
    }
    o_all += bk.nid;
  }
  XNS_TRY(xns_timer_stop(ctx));
  for (uint32_t e = 0; e < nel; e++) n_el[e] = (uint32_t)count[e];
  ctx->atoms_n.assign(n_el, n_el + nel);
  *xyz_dev = out;
  return XNS_OK;
}

extern "C" int xns_copy_atoms(xns_ctx *ctx, double *const *xyz_el) {
  if (!ctx) return XNS_ERR_ARG;
  if (!xyz_el) return xns_fail(ctx, XNS_ERR_ARG, "xns_copy_atoms: xyz_el is NULL");
  if (ctx->atoms_n.empty()) return xns_fail(ctx, XNS_ERR_ARG, "xns_copy_atoms: nothing built yet");
  const double *src = (const double *)ctx->slot_ptr[SLOT_ATOMS];
  size_t o = 0;
  for (size_t e = 0; e < ctx->atoms_n.size(); e++) {
    const size_t n = ctx->atoms_n[e];
    if (n) {
      if (!xyz_el[e]) return xns_fail(ctx, XNS_ERR_ARG, "xns_copy_atoms: NULL array for a non-empty element");
      XNS_CUDA(ctx, cudaMemcpyAsync(xyz_el[e], src + 3 * o, 24 * n, cudaMemcpyDeviceToHost, ctx->stream));
    }
    o += n;
  }
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XNS_OK;
}
