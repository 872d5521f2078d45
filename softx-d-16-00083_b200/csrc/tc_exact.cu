// Exact-accumulation sinc transform on the BF16 tensor cores: integer digits (tcgen05 kind::f16).
//
//   G[c][q] = sum_k n_c[k] * sin(q r_k) / (q r_k + 1e-8),   r_k = (k + 0.5) * bin
//
// (the calcInt1DHist contraction, CalcFunctions.cpp:855-864).  The split-BF16 transform (tc_gemm.cu)
// accumulates real products in FP32, and its rounding grows with the running sum; at the low-q minima
// of a small particle's I(q) that sum is 1e5-1e6 times the result, which puts the error above 1e-4 of
// I(q).  Here both operands are written as small integers, which BF16 holds exactly (|x| <= 256):
//   S[q][k] = sum_{i<5}  d_i / (128 * 256^i),  d_i in [-128, 128]  (S in FP64; residual < 1e-12)
//   n[k]    = sum_{j<NH} e_j * 256^j,          e_j in [0, 255]     (counts < 2^(8 NH), exact)
//   G       = sum_{i,j} 256^(j-i) / 128 * (d_i . e_j)
// A product of digits is an integer below 2^15 (128 * 255 = 32640) and a level v = j - i gains at most
// min(4, NH) <= 4 of them per k, so over a chunk of CH_K = 128 k every partial sum is an integer below
// 128 * 4 * 32640 < 2^24 and the FP32 tensor-memory accumulator holds it exactly.  All 4*NH digit products are kept; products of one level share one
// accumulator (4 + NH - 1 levels of 64 columns), and every chunk the accumulators are read, combined
// in FP64 (Horner over the levels, exact: below 2^53) and added to per-thread FP64 sums, which go to
// the output with FP64 atomics when the CTA's part of an output tile ends.
//
// Tile 128 q x N columns x 64 k (N = 16 or 32 for the transform, 64 for the plane), one CTA per SM,
// 2 stages of {NA A-digit tiles, NB B-digit tiles}; warp 0 loads (cp.async.bulk), warp 1 issues the
// MMAs, warps 2-9 drain tensor memory.  For the sinc transform the A digits are not loaded: warps
// 10-13 compute them into the stage (one q row per thread: an FP64 sine by rotation from one sincos
// per row and k tile, the sinc by an FP64 reciprocal, the five digits in FP32 from a hi/lo split;
// a fence.proxy.async makes the writes visible to the tensor core before the row's mbarrier arrival),
// so the only HBM traffic is the count digits and the output.  The accumulators are double-buffered in tensor memory
// (2 x levels x N <= 512 columns), so the MMAs of one chunk run while the previous chunk is drained;
// with N <= 32 the two groups of four drain warps take alternate chunks (one buffer each), with N = 64
// each group drains 32 columns of every chunk.  Waits are bounded as in tc_gemm.cu.
#include <algorithm>

#include "tc_gemm.cuh"
#include "tc_ptx.cuh"

using namespace xns_ptx;

namespace {

constexpr int XM = 128, XK = 64;  // tile: q rows, k (one 128-byte swizzle row of BF16); N per scheme
// Digits of the sinc matrix.  Four leave 2.4e-10 per element, which at the deepest minima of a
// 2e5-atom sphere is 2e-5 of I(q) (the sum over ~3e5 bins of 1e5 counts each); five leave 1e-12.
constexpr int NDS = 5;
constexpr int XA = XM * XK * 2;            // 16 KB per S-digit tile
constexpr int XSTAGES = 2;
constexpr int CH_TILES = 2;                // k tiles per exact chunk (CH_K = 128)
constexpr int XTHREADS = 320;
constexpr int XDRAIN_THREADS = 256;              // warps 2-9
constexpr int XGEN_WARPS = 8;                    // sinc-digit producers (warps 10-17): a q row, half the k
constexpr int XTHREADS_GEN = XTHREADS + 32 * XGEN_WARPS;
constexpr uint32_t XTMEM_COLS = 512;

// A digit scheme: NA digit planes of the A operand, NB of the B operand, NL accumulator levels, and the
// level of the product of A digit i with B digit j (-1: dropped; 0 is the most significant level).
//   KIND 0 (sinc transform): A = sinc digits, B = count digits, every product kept, level
//          (NB-1) - (j - i);
//   KIND 1 (plane amplitude): A and B = cos / sin digits, products of level i + j < NL kept.
template <int NA_, int NB_, int NL_, int KIND, int N_>
struct Scheme {
  static constexpr int NA = NA_, NB = NB_, NL = NL_, N = N_;
  static constexpr int XB = N * XK * 2;  // bytes per B-digit tile
  static constexpr bool ALT = N <= 16;   // drain groups take alternate chunks (else split the columns)
  static constexpr int STAGE = NA * XA + NB * XB;
  static constexpr int SMEM = XSTAGES * STAGE + 1024;
  static_assert(N % 16 == 0 && N >= 16 && N <= 64, "N tile: 16, 32 or 64 columns");
  static_assert(2 * NL * N <= (int)XTMEM_COLS, "two buffers of levels must fit in tensor memory");
  static_assert(SMEM <= 232448, "stages must fit in shared memory");
  __host__ __device__ static constexpr int level(int i, int j) {
    return KIND == 0 ? (NB - 1) - (j - i) : (i + j < NL ? i + j : -1);
  }
};
template <int NH, int N>
using SincScheme = Scheme<NDS, NH, NDS + NH - 1, 0, N>;

struct XArgs {
  const uint8_t *A;  // NA digit planes of MT*KT tiles, plane stride a_plane bytes
  const uint8_t *B;  // NB digit planes of NT*KT tiles, plane stride b_plane bytes
  size_t a_plane, b_plane;
  uint32_t MT, NT, KT;
  double *out;
  uint32_t ldo, m_valid, n_valid;
  double scale;  // value of one unit of the Horner sum over the levels
  int *err;
  uint32_t ksplit;  // 0: stream-K over all units; else K parts per output tile (grid = parts x tiles)
  unsigned long long wait_ns;  // bound of every pipeline wait (WAIT_LIMIT_NS unless a test asked less)
  int no_loads;                // failure-path test (xns_inject_pipeline_stall): the loader issues nothing
  // sinc digits made on chip (GEN): the q mesh (m_valid rows), the bin width and the bins used
  const double *qv;
  double bin;
  uint32_t nh;
};

// Conversions between FP64 and FP32 by integer operations (no conversion-pipe instruction):
// d with its low 29 mantissa bits cleared (24 significant bits, truncated toward zero) ...
__device__ __forceinline__ double short_double(double d) {
  return __hiloint2double(__double2hiint(d), __double2loint(d) & (int)0xe0000000);
}
// ... exactly as FP32 (0 below the FP32 normal range) ...
__device__ __forceinline__ float f32_of_short(double d) {
  const unsigned h = (unsigned)__double2hiint(d), l = (unsigned)__double2loint(d), mag = h & 0x7fffffffu;
  const unsigned bits = ((mag - (896u << 20)) << 3) | (l >> 29) | (h & 0x80000000u);
  return __uint_as_float(mag < (897u << 20) ? (h & 0x80000000u) : bits);
}
// ... and a normal FP32 (or 0) exactly as FP64.
__device__ __forceinline__ double f64_of_f32(float f) {
  const unsigned b = __float_as_uint(f), mag = b & 0x7fffffffu;
  const unsigned hi = (mag ? (mag >> 3) + (896u << 20) : 0u) | (b & 0x80000000u);
  return __hiloint2double((int)hi, (int)(mag << 29));
}

// 1/d for 1e-30 < d < 1e30: the FP32 reciprocal of d truncated to FP32 (relative error below 2^-21)
// and two Newton steps in FP64, each squaring the relative error (to the FP64 rounding).
__device__ __forceinline__ double recip64(double d) {
  float rf;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rf) : "f"(f32_of_short(short_double(d))));
  double r = f64_of_f32(rf);
  double e = __fma_rn(-d, r, 1.0);
  r = __fma_rn(r, e, r);
  e = __fma_rn(-d, r, 1.0);
  return __fma_rn(r, e, r);
}

// The five balanced base-256 digits of x = 128 v (|v| <= 1) as BF16 bit patterns (upper halves):
// N = round(x 2^32) comes out of one FMA with 1.5 * 2^52 (the integer lands in the mantissa: low word
// N mod 2^32, the low 20 bits of the high word 2^19 + floor(N / 2^32)); adding 0x80808080 biases each
// of the four low bytes by 128 with the carries, so that byte j of the sum minus 128 is digit j and
// the carried high part is the top digit:  x = sum_{i<5} dig[i] 256^-i + e, |dig[i]| <= 128,
// |e| <= 2^-33.  A digit becomes an exact FP32 by planting its byte under the exponent of 2^23 and
// subtracting 2^23 + 128; its BF16 is then the upper half of those bits.  dig[0] is the top digit.
__device__ __forceinline__ void sinc_digits(double x, uint32_t *dig) {
  const double t = __fma_rn(x, 4294967296.0, 6755399441055744.0);
  const uint32_t lo = (uint32_t)__double2loint(t);
  const int hi = (__double2hiint(t) & 0xfffff) - (1 << 19);
  uint32_t lo2;
  int hi2;
  asm("add.cc.u32 %0, %2, 0x80808080;\n\taddc.s32 %1, %3, 0;" : "=r"(lo2), "=r"(hi2) : "r"(lo), "r"(hi));
  const float B = 8388736.0f;  // 2^23 + 128
  dig[0] = __float_as_uint(__int_as_float(0x4B000000 + hi2 + 128) - B);
#pragma unroll
  for (int j = 0; j < 4; j++)  // byte 3 - j of lo2 is digit 1 + j (the most significant first)
    dig[1 + j] = __float_as_uint(__uint_as_float(__byte_perm(lo2, 0x4B000000u, 0x7540u | (3 - j))) - B);
}

// The sinc digits of 32 consecutive bins kb .. kb + 31 of one q row (q = qm), 8 bins per call of
// chunk(), as the BF16 bit patterns of the five digit planes (one uint4 of 8 bins per plane).  Both the
// on-chip producers and the HBM-plane kernel make every (row, k tile, half) with this same sequence, so
// the two give identical digits: sin by rotation from an FP64 sincos at kb (drift over 32 bins
// ~1e-14), x = q r_k stepped by q bin, 1/(x + 1e-8) from rcp.approx plus two Newton steps at kb (and
// everywhere in the first k tile, where neighbouring x differ by factors up to 3), otherwise by three
// Newton steps from the previous bin's reciprocal (relative error of that start below 1/64).
struct SincRun {
  double sn, cs, x, r, sd, cd, qb;
  bool first_tile;
  __device__ __forceinline__ void init(double qm, double bin, uint32_t kb, double sd_, double cd_) {
    sd = sd_;
    cd = cd_;
    qb = qm * bin;
    x = ((kb + 0.5) * bin) * qm;  // qrij = rij * q[iq] (CalcFunctions.cpp:858-861)
    sincos(x, &sn, &cs);
    sn *= 128.0;
    cs *= 128.0;
    first_tile = kb < XK;
  }
  __device__ __forceinline__ void chunk(uint32_t c, uint4 *w) {
    uint32_t dig[NDS][8];
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const double den = x + 0.00000001;
      if (first_tile || (c == 0 && e == 0)) {
        r = recip64(den);
      } else {
        double er = __fma_rn(-den, r, 1.0);
        r = __fma_rn(r, er, r);
        er = __fma_rn(-den, r, 1.0);
        r = __fma_rn(r, er, r);
        er = __fma_rn(-den, r, 1.0);
        r = __fma_rn(r, er, r);
      }
      // the reference's sin(q r)/(q r + 1e-8), times 128
      uint32_t d5[NDS];
      sinc_digits(sn * r, d5);
#pragma unroll
      for (int d = 0; d < NDS; d++) dig[d][e] = d5[d];
      const double s1 = __fma_rn(sn, cd, cs * sd), c1 = __fma_rn(cs, cd, -(sn * sd));
      sn = s1;
      cs = c1;
      x += qb;
    }
#pragma unroll
    for (int d = 0; d < NDS; d++) {
      w[d].x = __byte_perm(dig[d][0], dig[d][1], 0x7632);
      w[d].y = __byte_perm(dig[d][2], dig[d][3], 0x7632);
      w[d].z = __byte_perm(dig[d][4], dig[d][5], 0x7632);
      w[d].w = __byte_perm(dig[d][6], dig[d][7], 0x7632);
    }
  }
};

__device__ __forceinline__ uint32_t chunk_offset(uint32_t row, uint32_t ch);

template <class E, bool GEN>
__global__ void __launch_bounds__(GEN ? XTHREADS_GEN : XTHREADS, 1) sinc_exact_kernel(const XArgs g) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) unsigned long long bars[2 * XSTAGES + 5];
  __shared__ uint32_t tmem_sh;
  __shared__ int abort_sh;
  const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
  const uint32_t full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[XSTAGES]);
  // per accumulator buffer b: tfull0 + 8 b (MMAs done), tempty0 + 8 b (drained)
  const uint32_t tfull0 = smem_u32(&bars[2 * XSTAGES]), tempty0 = smem_u32(&bars[2 * XSTAGES + 2]);
  const uint32_t drain = smem_u32(&bars[2 * XSTAGES + 4]);
  constexpr uint32_t BUFCOLS = E::NL * E::N;  // tensor-memory columns of one accumulator buffer
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  volatile int *abort = &abort_sh;

  if (threadIdx.x == 0) {
    for (int s = 0; s < XSTAGES; s++) {
      mbar_init(full0 + 8 * s, GEN ? 1 + 32 * XGEN_WARPS : 1);  // the copy warp (+ every producer thread)
      mbar_init(empty0 + 8 * s, 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(tfull0 + 8 * b, 1);
      mbar_init(tempty0 + 8 * b, E::ALT ? 128 : XDRAIN_THREADS);
    }
    mbar_init(drain, 1);
    abort_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_sh)),
                 "r"(XTMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_sh;

  const unsigned long long KT = g.KT;
  const unsigned long long units = (unsigned long long)g.NT * g.MT * KT;
  // ksplit 0: the units are cut into gridDim.x equal ranges (stream-K); ksplit > 0: CTA b takes K part
  // b / tiles of output tile b % tiles (CTAs that run together work on the same K part)
  unsigned long long u0, u1;
  if (g.ksplit) {
    const unsigned long long tiles = (unsigned long long)g.NT * g.MT, t = blockIdx.x % tiles, kq = blockIdx.x / tiles;
    u0 = t * KT + KT * kq / g.ksplit;
    u1 = t * KT + KT * (kq + 1) / g.ksplit;
  } else {
    u0 = units * blockIdx.x / gridDim.x;
    u1 = units * (blockIdx.x + 1) / gridDim.x;
  }

  if (warp == 0) {
    if (lane == 0) {  // loader
      uint32_t fills[XSTAGES] = {};
      unsigned long long i = 0;
      for (unsigned long long u = g.no_loads ? u1 : u0; u < u1; ++u, ++i) {
        const uint32_t s = (uint32_t)(i % XSTAGES), k = (uint32_t)(i / XSTAGES);
        if (k > 0 && !mbar_wait(empty0 + 8 * s, (k - 1) & 1u, abort, g.wait_ns)) {
          abort_sh = 1;
          atomicOr(g.err, 1);
          break;
        }
        const uint32_t kt = (uint32_t)(u % KT);
        const unsigned long long r = u / KT;
        const uint32_t mt = (uint32_t)(r % g.MT), nt = (uint32_t)(r / g.MT);
        const uint32_t dst = base + s * E::STAGE, bar = full0 + 8 * s;
        const size_t ao = ((size_t)mt * g.KT + kt) * XA, bo = ((size_t)nt * g.KT + kt) * E::XB;
        mbar_expect_tx(bar, (uint32_t)(GEN ? E::NB * E::XB : E::STAGE));
        if (!GEN) {
#pragma unroll
          for (int d = 0; d < E::NA; d++) bulk_g2s(dst + d * XA, g.A + d * g.a_plane + ao, XA, bar);
        }
#pragma unroll
        for (int e = 0; e < E::NB; e++) bulk_g2s(dst + E::NA * XA + e * E::XB, g.B + e * g.b_plane + bo, E::XB, bar);
        fills[s] = k + 1;
      }
      if (*abort)
        for (int s = 0; s < XSTAGES; s++)
          if (fills[s]) mbar_wait(full0 + 8 * s, (fills[s] - 1) & 1u, nullptr, DRAIN_LIMIT_NS);
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      // kind::f16: F32 accumulator (1), BF16 A and B (1, 1), K-major, N = E::N, M = 128
      const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(E::N >> 3) << 17) | ((uint32_t)(XM >> 4) << 24);
      uint32_t chunk = 0;  // chunks handed to the drain warps so far
      bool issued = false;
      unsigned long long i = 0;
      uint32_t in_chunk = 0;
      for (unsigned long long u = u0; u < u1; ++u, ++i) {
        const uint32_t s = (uint32_t)(i % XSTAGES), k = (uint32_t)(i / XSTAGES);
        const bool seg_first = (u == u0) || (u % KT == 0);
        const bool seg_last = (u + 1 == u1) || ((u + 1) % KT == 0);
        const bool first = seg_first || in_chunk == 0;
        if (first && chunk >= 2) {  // the drain warps have read this buffer's previous chunk
          if (!mbar_wait(tempty0 + 8 * (chunk & 1u), ((chunk >> 1) - 1) & 1u, abort, g.wait_ns)) {
            abort_sh = 1;
            atomicOr(g.err, 1);
            break;
          }
          tc_fence_after();
        }
        if (!mbar_wait(full0 + 8 * s, k & 1u, abort, g.wait_ns)) {
          abort_sh = 1;
          atomicOr(g.err, 1);
          break;
        }
        tc_fence_after();
        const uint32_t a0 = base + s * E::STAGE, b0 = a0 + E::NA * XA, tacc = tmem + (chunk & 1u) * BUFCOLS;
#pragma unroll
        for (int ks = 0; ks < XK / 16; ks++) {
          const uint32_t off = ks * 32;
          uint32_t written = 0;
#pragma unroll
          for (int di = 0; di < E::NA; di++) {
#pragma unroll
            for (int ej = 0; ej < E::NB; ej++) {
              const int lev = E::level(di, ej);  // 0 = top level
              if (lev < 0) continue;
              const uint32_t acc = (first && ks == 0 && !(written & (1u << lev))) ? 0u : 1u;
              written |= 1u << lev;
              tc_mma(tacc + lev * E::N, sw128_desc(a0 + di * XA + off), sw128_desc(b0 + ej * E::XB + off), idesc, acc);
            }
          }
        }
        issued = true;
        tc_commit(empty0 + 8 * s);
        in_chunk++;
        if (seg_last || in_chunk == CH_TILES) {
          tc_commit(tfull0 + 8 * (chunk & 1u));
          chunk++;
          in_chunk = 0;
        }
      }
      if (*abort && issued) {
        tc_commit(drain);
        mbar_wait(drain, 0, nullptr, DRAIN_LIMIT_NS);
      }
    }
  } else if (warp < 10) {
    // drain: warp w reads TMEM lanes 32*(w%4) .. +31 (its quarter of the 128 rows).  Group h = 0, 1:
    // with ALT, chunks c with c % 2 == h (buffer h), all N columns; otherwise every chunk, columns
    // h N/2 .. (h + 1) N/2 - 1.
    constexpr int COLS = E::ALT ? E::N : E::N / 2;
    const uint32_t wq = warp & 3, h = (uint32_t)(warp - 2) >> 2;
    const uint32_t lane_addr = tmem + ((wq * 32u) << 16) + (E::ALT ? 0u : h * (uint32_t)COLS);
    double sum[COLS];
#pragma unroll
    for (int j = 0; j < COLS; j++) sum[j] = 0.0;
    uint32_t chunk = 0, in_chunk = 0;
    for (unsigned long long u = u0; u < u1; ++u) {
      const bool seg_last = (u + 1 == u1) || ((u + 1) % KT == 0);
      in_chunk++;
      if (!(seg_last || in_chunk == CH_TILES)) continue;
      in_chunk = 0;
      const uint32_t b = chunk & 1u;
      if (!E::ALT || b == h) {
        const bool ok = mbar_wait(tfull0 + 8 * b, (chunk >> 1) & 1u, abort, g.wait_ns);
        if (__any_sync(0xffffffffu, !ok)) {
          abort_sh = 1;
          if (lane == 0) atomicOr(g.err, 1);
          break;
        }
        tc_fence_after();
#pragma unroll
        for (int c = 0; c < COLS; c += 8) {
          double t[8];
#pragma unroll
          for (int j = 0; j < 8; j++) t[j] = 0.0;
#pragma unroll
          for (int lev = 0; lev < E::NL; lev++) {  // Horner over the levels, top first
            uint32_t rr[8];
            tc_ld8_raw(lane_addr + b * BUFCOLS + lev * E::N + c, rr);
#pragma unroll
            for (int j = 0; j < 8; j++) t[j] = t[j] * 256.0 + (double)__uint_as_float(rr[j]);
          }
#pragma unroll
          for (int j = 0; j < 8; j++) sum[c + j] += t[j];
        }
        tc_fence_before();
        mbar_arrive(tempty0 + 8 * b);
      }
      chunk++;
      if (seg_last) {
        const unsigned long long r = u / KT;
        const uint32_t mt = (uint32_t)(r % g.MT), nt = (uint32_t)(r / g.MT);
        const uint32_t m = mt * XM + wq * 32 + lane;
        const double scale = g.scale;
        if (m < g.m_valid) {
#pragma unroll
          for (int j = 0; j < COLS; j++) {
            const uint32_t n = nt * E::N + (E::ALT ? 0u : h * (uint32_t)COLS) + j;
            if (n < g.n_valid && sum[j] != 0.0) atomicAdd(g.out + (size_t)n * g.ldo + m, sum[j] * scale);
          }
        }
#pragma unroll
        for (int j = 0; j < COLS; j++) sum[j] = 0.0;
      }
    }
  }
  if (GEN && warp >= 10) {
    // sinc-digit producers: thread t makes q row t % 128, bins 32 (t / 128) .. +31 of every A tile of
    // this CTA's units (SincRun: the same digits as the HBM planes)
    const uint32_t t = (uint32_t)(warp - 10) * 32u + lane, row = t & 127u, half = t >> 7;
    uint8_t *gsm = smem_raw + (base - smem_u32(smem_raw));
    uint32_t cur_mt = 0xffffffffu;
    double qm = 0.0, sd = 0.0, cd = 1.0;
    unsigned long long i = 0;
    for (unsigned long long u = u0; u < u1; ++u, ++i) {
      const uint32_t s = (uint32_t)(i % XSTAGES), k = (uint32_t)(i / XSTAGES);
      if (k > 0 && !mbar_wait(empty0 + 8 * s, (k - 1) & 1u, abort, g.wait_ns)) {
        abort_sh = 1;
        atomicOr(g.err, 1);
        break;
      }
      const uint32_t kt = (uint32_t)(u % KT), mt = (uint32_t)((u / KT) % g.MT);
      if (mt != cur_mt) {  // rows past the mesh have q = 0: zero digits
        const uint32_t m = mt * XM + row;
        qm = m < g.m_valid ? g.qv[m] : 0.0;
        sincos(qm * g.bin, &sd, &cd);
        cur_mt = mt;
      }
      SincRun run;
      run.init(qm, g.bin, kt * XK + 32u * half, sd, cd);
      uint8_t *st = gsm + s * E::STAGE;
#pragma unroll 1
      for (uint32_t c = 0; c < 4; c++) {
        uint4 w[NDS];
        run.chunk(c, w);
        const uint32_t off = chunk_offset(row, 4u * half + c);
#pragma unroll
        for (int d = 0; d < NDS; d++) *(uint4 *)(st + d * XA + off) = w[d];
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes -> tensor-core reads
      mbar_arrive(full0 + 8 * s);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(XTMEM_COLS) : "memory");
}

// Byte offset of the 16-byte chunk ch of row `row` in a K-major 128-byte-swizzled tile.
__device__ __forceinline__ uint32_t chunk_offset(uint32_t row, uint32_t ch) {
  return (row >> 3) * 1024u + (row & 7u) * 128u + (((ch ^ row) & 7u) << 4);
}

__device__ __forceinline__ uint4 pack8(const float *v) {
  __align__(16) __nv_bfloat16 b[8];
#pragma unroll
  for (int i = 0; i < 8; i++) b[i] = __float2bfloat16_rn(v[i]);  // integers |v| <= 256: exact
  return *(const uint4 *)b;
}

// The sinc digits as planes in HBM, for a q mesh used again (streamed by the copy warp instead of made
// on chip; SincRun makes the same digits).  One CTA of 256 threads per (mt, kt) tile: thread t makes
// row t % 128, bins 32 (t / 128) .. +31.
__global__ void pack_sinc_digits_kernel(const double *__restrict__ q, uint32_t nq, double bin, uint32_t KT,
                                        uint8_t *__restrict__ A, size_t a_plane) {
  const uint32_t tile = blockIdx.x, mt = tile / KT, kt = tile % KT;
  const uint32_t row = threadIdx.x & 127u, half = threadIdx.x >> 7, m = mt * XM + row;
  const double qm = m < nq ? q[m] : 0.0;
  double sd, cd;
  sincos(qm * bin, &sd, &cd);
  SincRun run;
  run.init(qm, bin, kt * XK + 32u * half, sd, cd);
  for (uint32_t c = 0; c < 4; c++) {
    uint4 w[NDS];
    run.chunk(c, w);
    const size_t off = (size_t)tile * XA + chunk_offset(row, 4u * half + c);
#pragma unroll
    for (int d = 0; d < NDS; d++) *(uint4 *)(A + d * a_plane + off) = w[d];
  }
}

// One CTA per (nt, kt) tile of N rows (histogram columns).  Sets *overflow when a count needs more
// than NH digits.
template <int NH, int N>
__global__ void pack_count_digits_kernel(const unsigned long long *__restrict__ hist, uint32_t ncols, uint32_t nh,
                                         size_t ldh, uint32_t KT, uint8_t *__restrict__ B, size_t b_plane,
                                         int *overflow) {
  const uint32_t tile = blockIdx.x, nt = tile / KT, kt = tile % KT;
  for (uint32_t c = threadIdx.x; c < N * 8; c += blockDim.x) {
    const uint32_t row = c >> 3, ch = c & 7, n = nt * N + row, k0 = kt * XK + ch * 8;
    float dig[NH][8];
    bool big = false;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const uint32_t k = k0 + i;
      const unsigned long long v = (n < ncols && k < nh) ? hist[(size_t)n * ldh + k] : 0ull;
      big |= (v >> (8 * NH)) != 0;
#pragma unroll
      for (int e = 0; e < NH; e++) dig[e][i] = (float)((v >> (8 * e)) & 255u);
    }
    if (big) atomicOr(overflow, 1);
    const size_t off = (size_t)tile * (N * XK * 2) + chunk_offset(row, ch);
#pragma unroll
    for (int e = 0; e < NH; e++) *(uint4 *)(B + e * b_plane + off) = pack8(dig[e]);
  }
}

__global__ void max_count_kernel(const unsigned long long *__restrict__ hist, uint32_t ncols, uint32_t nh, size_t ldh,
                                 unsigned long long *out) {
  unsigned long long m = 0;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < (size_t)ncols * nh; t += (size_t)gridDim.x * blockDim.x)
    m = max(m, hist[(t / nh) * ldh + t % nh]);
  for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

// Launches the digit GEMM of scheme E; grid 0: one CTA per SM (stream-K over all units), otherwise the
// given number of CTAs.
template <class E, bool GEN>
int launch_digit_gemm(xns_ctx *ctx, const XArgs &g0, unsigned grid) {
  XArgs g = g0;
  g.wait_ns = ctx->inject_stall_ns ? ctx->inject_stall_ns : WAIT_LIMIT_NS;
  g.no_loads = ctx->inject_stall_ns != 0;
  ctx->inject_stall_ns = 0;  // one call only
  static bool attr_set[XNS_MAX_DEVICES] = {};  // the attribute is per device; set once on each
  if (ctx->device < 0 || ctx->device >= XNS_MAX_DEVICES || !attr_set[ctx->device]) {
    XNS_CUDA(ctx, cudaFuncSetAttribute(sinc_exact_kernel<E, GEN>, cudaFuncAttributeMaxDynamicSharedMemorySize, E::SMEM));
    if (ctx->device >= 0 && ctx->device < XNS_MAX_DEVICES) attr_set[ctx->device] = true;
  }
  const unsigned long long units = (unsigned long long)g.NT * g.MT * g.KT;
  if (!grid) grid = (unsigned)std::min<unsigned long long>((unsigned long long)ctx->num_sms, units);
  sinc_exact_kernel<E, GEN><<<grid, GEN ? XTHREADS_GEN : XTHREADS, E::SMEM, ctx->stream>>>(g);
  XNS_LAUNCHED(ctx);
  return XNS_OK;
}

template <int NH, int N>
int enqueue_exact(xns_ctx *ctx, const ExactLaunch &X) {
  pack_count_digits_kernel<NH, N><<<X.NT * X.KT, 256, 0, ctx->stream>>>(X.hist, X.ncols, X.nh, X.ldh, X.KT, X.B,
                                                                         X.b_plane, X.flags + 1);
  XNS_LAUNCHED(ctx);
  XArgs g{};
  g.A = X.A;  // null: made on chip
  g.B = X.B;
  g.a_plane = X.a_plane;
  g.b_plane = X.b_plane;
  g.qv = X.qv;
  g.bin = X.bin;
  g.nh = X.nh;
  g.MT = X.MT;
  g.NT = X.NT;
  g.KT = X.KT;
  g.out = X.G;
  g.ldo = X.nq;
  g.m_valid = X.nq;
  g.n_valid = X.ncols;
  g.err = X.flags;
  // level l holds 256^(NH-1-l)/128; the Horner sum weights it 256^(NL-1-l): one unit is 256^-(NDS-1)/128
  g.scale = ldexp(1.0, -8 * (NDS - 1)) / 128.0;
  return X.A ? launch_digit_gemm<SincScheme<NH, N>, false>(ctx, g, 0) : launch_digit_gemm<SincScheme<NH, N>, true>(ctx, g, 0);
}

template <int NH>
int enqueue_exact_n(xns_ctx *ctx, const ExactLaunch &X) {
  return X.ntile == 16 ? enqueue_exact<NH, 16>(ctx, X) : enqueue_exact<NH, 32>(ctx, X);
}

// ---- 2D amplitude on a Cartesian q plane ---------------------------------------------------------
//
// A_e(qx, qy) = sum_{j in e} exp(i (qx x_j + qy y_j)) factorises into cos / sin of qx x_j and qy y_j,
// so Re A_e and Im A_e are one real GEMM over k = 2 n_e: A rows are qx with columns
// [cos(qx x_j) | sin(qx x_j)], B rows are first qy for Re with [cos(qy y_j) | -sin(qy y_j)], then qy for
// Im with [sin(qy y_j) | cos(qy y_j)].  Values in [-1, 1] (FP64 sines) become PD base-256 digits
// (d/128 + d'/128/256 + ...) and the digit products of level i + j < PD are summed exactly
// (PlaneScheme).  Three digits (residual 2^-24) leave 1e-5..3e-5 of I at the dim points of a crystal's
// pattern, where the rounding of the lattice's repeated phases adds coherently; four leave 2^-32.
constexpr int PD = 4;
constexpr int PN = 64;                 // plane: B tile rows (qy rows for Re, then for Im)
constexpr int PXB = PN * XK * 2;
using PlaneScheme = Scheme<PD, PD, PD, 1, PN>;

__device__ __forceinline__ void put_digits(uint8_t *plane0, size_t plane, size_t off, double v) {
  double r = v * 128.0;
#pragma unroll
  for (int d = 0; d < PD; d++) {
    const double di = rint(r);
    *reinterpret_cast<__nv_bfloat16 *>(plane0 + d * plane + off) = __float2bfloat16_rn((float)di);
    r = (r - di) * 256.0;
  }
}

// One CTA of 64 threads per (mt, kt) tile of the qx operand; thread = column k; the 128 rows come from
// one FP64 sincos and the rotation by dq x (FP64, drift ~1e-14 over 128 rows).
__global__ void plane_pack_a_kernel(const double *__restrict__ x, uint32_t n, double q0, double dq, uint32_t nq,
                                    uint32_t KT, uint8_t *__restrict__ A, size_t a_plane) {
  const uint32_t tile = blockIdx.x, mt = tile / KT, kt = tile % KT, kk = threadIdx.x, k = kt * XK + kk;
  const bool use = k < 2 * n, is_sin = k >= n;
  const double xj = use ? x[is_sin ? k - n : k] : 0.0;
  double s, c, sd, cd;
  sincos((q0 + (double)(mt * XM) * dq) * xj, &s, &c);
  sincos(dq * xj, &sd, &cd);
  uint8_t *t0 = A + (size_t)tile * XA;
  for (uint32_t row = 0; row < XM; row++) {
    const bool valid = use && mt * XM + row < nq;
    put_digits(t0, a_plane, xns_tc::sw128_offset(row, kk), valid ? (is_sin ? s : c) : 0.0);
    const double s1 = fma(s, cd, c * sd), c1 = fma(c, cd, -(s * sd));
    s = s1;
    c = c1;
  }
}

// One CTA of 64 threads per (nt, kt) tile of the qy operand (rows: qy for Re, then qy for Im).
__global__ void plane_pack_b_kernel(const double *__restrict__ y, uint32_t n, double q0, double dq, uint32_t nq,
                                    uint32_t KT, uint8_t *__restrict__ B, size_t b_plane) {
  const uint32_t tile = blockIdx.x, nt = tile / KT, kt = tile % KT, kk = threadIdx.x, k = kt * XK + kk;
  const bool use = k < 2 * n, second = k >= n;
  const double yj = use ? y[second ? k - n : k] : 0.0;
  double s = 0, c = 1, sd, cd;
  sincos(dq * yj, &sd, &cd);
  uint8_t *t0 = B + (size_t)tile * PXB;
  for (uint32_t row = 0; row < PN; row++) {
    const uint32_t np = nt * PN + row, part = np >= nq ? 1u : 0u, iy = np - part * nq;
    if (row == 0 || iy == 0) sincos((q0 + (double)iy * dq) * yj, &s, &c);  // new run of qy
    double v = 0.0;
    if (use && np < 2 * nq) v = part == 0 ? (second ? -s : c) : (second ? c : s);
    put_digits(t0, b_plane, xns_tc::sw128_offset(row, kk), v);
    const double s1 = fma(s, cd, c * sd), c1 = fma(c, cd, -(s * sd));
    s = s1;
    c = c1;
  }
}

// Ar/Ai (nqy x nqx) += f_e(|q|) * (Re, Im) of one element; f from 4-Gaussian coefficients (X-ray) or a
// scattering length.
__global__ void plane_accum_kernel(const double *__restrict__ C, uint32_t nqx, uint32_t nqy, double qx0, double dqx,
                                   double qy0, double dqy, const double *__restrict__ coef, double sl,
                                   double *__restrict__ Ar, double *__restrict__ Ai) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)nqx * nqy) return;
  const uint32_t iy = (uint32_t)(i / nqx), ix = (uint32_t)(i % nqx);
  double f = sl;
  if (coef) {
    const double qx = qx0 + ix * dqx, qy = qy0 + iy * dqy, qm = sqrt(qx * qx + qy * qy);
    const double s2 = (qm / (4.0 * XNS_PI)) * (qm / (4.0 * XNS_PI));
    f = coef[0] * exp(-coef[4] * s2) + coef[1] * exp(-coef[5] * s2) + coef[2] * exp(-coef[6] * s2) +
        coef[3] * exp(-coef[7] * s2) + coef[8];
  }
  Ar[i] += f * C[(size_t)iy * nqx + ix];
  Ai[i] += f * C[(size_t)(nqy + iy) * nqx + ix];
}

__global__ void plane_intensity_kernel(const double *__restrict__ Ar, const double *__restrict__ Ai, size_t n, double inv_n,
                                       double *__restrict__ I) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) I[i] = (Ar[i] * Ar[i] + Ai[i] * Ai[i]) * inv_n;
}

}  // namespace

int xns_tc_exact_plan(xns_ctx *ctx, const unsigned long long *d_hist, uint32_t ncols, uint32_t nh, size_t ldh, double bin,
                      const double *q, uint32_t nq, unsigned long long max_count, double *d_G, ExactLaunch *X,
                      bool planes) {
  *X = ExactLaunch();
  if (!ncols || !nq) return XNS_OK;
  if (max_count >> 32) return xns_fail(ctx, XNS_ERR_LIMIT, "exact transform: a bin count reaches 2^32");
  X->digits = (max_count >> 24) ? 4 : (max_count >> 16) ? 3 : 2;
  X->hist = d_hist;
  X->ncols = ncols;
  X->nh = nh;
  X->ldh = ldh;
  X->nq = nq;
  X->G = d_G;
  X->MT = (nq + XM - 1) / XM;
  X->KT = (nh + XK - 1) / XK;
  // narrow N tiles: the accumulators of two chunks must fit in tensor memory (2 x levels x N <= 512)
  X->ntile = ncols <= 16 ? 16 : 32;
  X->NT = (ncols + X->ntile - 1) / X->ntile;
  int st;
  void *flags;
  if ((st = xns_scratch(ctx, SLOT_FLAGS, 64, &flags))) return st;
  X->flags = (int *)flags;
  // the q mesh on the device (the sinc digits are made on chip from it)
  void *dq;
  if ((st = xns_scratch(ctx, SLOT_X_Q, sizeof(double) * nq, &dq))) return st;
  XNS_CUDA(ctx, cudaMemcpyAsync(dq, q, sizeof(double) * nq, cudaMemcpyHostToDevice, ctx->stream));
  X->qv = (const double *)dq;
  X->bin = bin;
  // A mesh seen for the first time gets its sinc digits made on chip (4.5 ms at 4096 q x 2.9e5 bins,
  // no HBM planes); a mesh used again (or when the caller asks, as a batch replayed from a graph does)
  // gets them as planes in HBM, made once (11.9 GB, 12 ms there) and streamed at copy bandwidth on every
  // call (2.4 ms).  A memory limit that the planes would exceed keeps the digits on chip.
  const size_t a_plane = (size_t)X->MT * X->KT * XA;
  auto same_mesh = [&](const std::vector<double> &mq, double mbin, uint32_t mkt) {
    return mbin == bin && mkt == X->KT && mq.size() == nq && std::equal(q, q + nq, mq.begin());
  };
  const bool cached = same_mesh(ctx->x_q, ctx->x_bin, ctx->x_kt) && ctx->slot_size[SLOT_X_A] >= NDS * a_plane;
  bool want = cached || planes || same_mesh(ctx->x_seen_q, ctx->x_seen_bin, ctx->x_seen_kt);
  if (want && !cached && ctx->mem_limit) {
    size_t others = 0;
    for (int k = 0; k < SLOT_COUNT; k++)
      if (k != SLOT_X_A) others += ctx->slot_size[k];
    want = others + NDS * a_plane <= ctx->mem_limit;
  }
  ctx->x_seen_q.assign(q, q + nq);
  ctx->x_seen_bin = bin;
  ctx->x_seen_kt = X->KT;
  void *A = nullptr;
  if (want && (st = xns_scratch(ctx, SLOT_X_A, NDS * a_plane, &A))) {
    if (st != XNS_ERR_NOMEM) return st;
    want = false;  // no room for the planes: the digits stay on chip
    ctx->err.clear();
  }
  if (want) {
    if (!cached) {
      pack_sinc_digits_kernel<<<X->MT * X->KT, 2 * XM, 0, ctx->stream>>>((const double *)dq, nq, bin, X->KT,
                                                                          (uint8_t *)A, a_plane);
      XNS_LAUNCHED(ctx);
      ctx->x_q.assign(q, q + nq);
      ctx->x_bin = bin;
      ctx->x_kt = X->KT;
    }
    X->A = (const uint8_t *)A;
    X->a_plane = a_plane;
  }
  X->b_plane = (size_t)X->NT * X->KT * X->ntile * XK * 2;
  void *B;
  if ((st = xns_scratch(ctx, SLOT_TC_B, X->digits * X->b_plane, &B))) return st;
  X->B = (uint8_t *)B;
  return XNS_OK;
}

int xns_tc_exact_enqueue(xns_ctx *ctx, const ExactLaunch &X) {
  if (!X.ncols) return XNS_OK;
  XNS_CUDA(ctx, cudaMemsetAsync(X.flags, 0, 2 * sizeof(int), ctx->stream));
  XNS_CUDA(ctx, cudaMemsetAsync(X.G, 0, sizeof(double) * X.ncols * X.nq, ctx->stream));
  switch (X.digits) {
    case 2: return enqueue_exact_n<2>(ctx, X);
    case 3: return enqueue_exact_n<3>(ctx, X);
    default: return enqueue_exact_n<4>(ctx, X);
  }
}

int xns_tc_exact_check(xns_ctx *ctx, const ExactLaunch &X) {
  if (!X.ncols) return XNS_OK;
  int err[2] = {0, 0};
  XNS_CUDA(ctx, cudaMemcpyAsync(err, X.flags, sizeof(err), cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (err[0]) return xns_fail(ctx, XNS_ERR_CUDA, "exact transform: a pipeline wait ran out of time");
  if (err[1]) return xns_fail(ctx, XNS_ERR_LIMIT, "exact transform: a bin count exceeds the planned digits");
  return XNS_OK;
}

int xns_tc_max_count(xns_ctx *ctx, const unsigned long long *d_hist, uint32_t ncols, uint32_t nh, size_t ldh,
                     unsigned long long *max_count) {
  int st;
  void *flags;
  if ((st = xns_scratch(ctx, SLOT_FLAGS, 64, &flags))) return st;
  unsigned long long *d_max = (unsigned long long *)((char *)flags + 8);
  XNS_CUDA(ctx, cudaMemsetAsync(d_max, 0, 8, ctx->stream));
  max_count_kernel<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(d_hist, ncols, nh, ldh, d_max);
  XNS_LAUNCHED(ctx);
  XNS_CUDA(ctx, cudaMemcpyAsync(max_count, d_max, 8, cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XNS_OK;
}

int xns_tc_hist_transform_exact(xns_ctx *ctx, const unsigned long long *d_hist, uint32_t ncols, uint32_t nh, size_t ldh,
                                double bin, const double *q, uint32_t nq, double *d_G) {
  if (!ncols || !nq) return XNS_OK;
  int st;
  unsigned long long maxc = 0;  // the largest count picks the number of count digits
  if ((st = xns_tc_max_count(ctx, d_hist, ncols, nh, ldh, &maxc))) return st;
  ExactLaunch X;
  if ((st = xns_tc_exact_plan(ctx, d_hist, ncols, nh, ldh, bin, q, nq, maxc, d_G, &X))) return st;
  if ((st = xns_tc_exact_enqueue(ctx, X))) return st;
  return xns_tc_exact_check(ctx, X);
}

// Host-buffer entry: as xns_hist_transform_bf16x3, with exact digit accumulation.
extern "C" int xns_hist_transform_exact(xns_ctx *ctx, const uint64_t *hist, uint32_t ncols, uint32_t nh, double bin,
                                        const double *q, uint32_t nq, double *G) {
  if (!ctx) return XNS_ERR_ARG;
  if (!hist || !q || !G || !ncols || !nh || !nq) return xns_fail(ctx, XNS_ERR_ARG, "transform: null or empty argument");
  int st;
  void *dh, *dG;
  if ((st = xns_scratch(ctx, SLOT_HIST, sizeof(uint64_t) * ncols * nh, &dh))) return st;
  if ((st = xns_scratch(ctx, SLOT_TC_OUT, sizeof(double) * ncols * nq, &dG))) return st;
  XNS_CUDA(ctx, cudaMemcpyAsync(dh, hist, sizeof(uint64_t) * ncols * nh, cudaMemcpyHostToDevice, ctx->stream));
  if ((st = xns_timer_start(ctx))) return st;
  if ((st = xns_stage_begin(ctx, STAGE_IQ))) return st;
  if ((st = xns_tc_hist_transform_exact(ctx, (const unsigned long long *)dh, ncols, nh, nh, bin, q, nq, (double *)dG)))
    return st;
  if ((st = xns_stage_end(ctx, STAGE_IQ))) return st;
  if ((st = xns_timer_stop(ctx))) return st;
  XNS_CUDA(ctx, cudaMemcpyAsync(G, dG, sizeof(double) * ncols * nq, cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XNS_OK;
}

// I[iy * nqx + ix] = |sum_e f_e(|q|) sum_{j in e} exp(i (qx x_j + qy y_j))|^2 / N on the plane
// qx = qx0 + ix dqx, qy = qy0 + iy dqy (coordinates as given: rotate them first for another
// orientation).  coef: 9 coefficients per element (X-ray) or null with sl (neutron).
extern "C" int xns_calc_amp_plane(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel,
                                  double qx0, double dqx, uint32_t nqx, double qy0, double dqy, uint32_t nqy, int source,
                                  const double *coef, const double *sl, double *I) {
  if (!ctx) return XNS_ERR_ARG;
  if (!I || nqx == 0 || nqy == 0) return xns_fail(ctx, XNS_ERR_ARG, "plane: null output or empty mesh");
  if (source == XNS_XRAY ? !coef : !sl) return xns_fail(ctx, XNS_ERR_ARG, "plane: missing form factors / lengths");
  int st;
  DevCoords dc;
  if ((st = xns_upload_coords(ctx, xyz_el, n_el, nel, &dc))) return st;
  if (dc.ntot == 0) return xns_fail(ctx, XNS_ERR_ARG, "plane: no atoms");
  const size_t npix = (size_t)nqx * nqy;
  void *vacc, *vC, *vI, *vcoef = nullptr, *flags;
  if ((st = xns_scratch(ctx, SLOT_OUT, sizeof(double) * 2 * npix, &vacc))) return st;
  if ((st = xns_scratch(ctx, SLOT_TC_OUT, sizeof(double) * 2 * npix, &vC))) return st;
  if ((st = xns_scratch(ctx, SLOT_OUT2, sizeof(double) * npix, &vI))) return st;
  if ((st = xns_scratch(ctx, SLOT_FLAGS, 64, &flags))) return st;
  if (source == XNS_XRAY) {
    if ((st = xns_scratch(ctx, SLOT_WEIGHTS, sizeof(double) * 9 * nel, &vcoef))) return st;
    XNS_CUDA(ctx, cudaMemcpyAsync(vcoef, coef, sizeof(double) * 9 * nel, cudaMemcpyHostToDevice, ctx->stream));
  }
  double *Ar = (double *)vacc, *Ai = Ar + npix;
  if ((st = xns_timer_start(ctx))) return st;
  if ((st = xns_stage_begin(ctx, STAGE_2D))) return st;
  XNS_CUDA(ctx, cudaMemsetAsync(vacc, 0, sizeof(double) * 2 * npix, ctx->stream));
  XNS_CUDA(ctx, cudaMemsetAsync(flags, 0, sizeof(int), ctx->stream));
  const uint32_t MT = (nqx + XM - 1) / XM, NT = (2 * nqy + PN - 1) / PN;
  for (uint32_t e = 0; e < nel; e++) {
    const uint32_t n = dc.n_el[e];
    if (!n) continue;
    const uint32_t KT = (2 * n + XK - 1) / XK;
    const size_t a_plane = (size_t)MT * KT * XA, b_plane = (size_t)NT * KT * PXB;
    void *A, *B;
    if ((st = xns_scratch(ctx, SLOT_X_A, PD * a_plane, &A))) return st;
    ctx->x_q.clear();  // the sinc-digit planes of the histogram transform share SLOT_X_A
    if ((st = xns_scratch(ctx, SLOT_TC_B, PD * b_plane, &B))) return st;
    const double *xe = dc.x + dc.off_el[e], *ye = dc.y + dc.off_el[e];
    plane_pack_a_kernel<<<MT * KT, XK, 0, ctx->stream>>>(xe, n, qx0, dqx, nqx, KT, (uint8_t *)A, a_plane);
    XNS_LAUNCHED(ctx);
    plane_pack_b_kernel<<<NT * KT, XK, 0, ctx->stream>>>(ye, n, qy0, dqy, nqy, KT, (uint8_t *)B, b_plane);
    XNS_LAUNCHED(ctx);
    XNS_CUDA(ctx, cudaMemsetAsync(vC, 0, sizeof(double) * 2 * npix, ctx->stream));
    XArgs g{};
    g.A = (const uint8_t *)A;
    g.B = (const uint8_t *)B;
    g.a_plane = a_plane;
    g.b_plane = b_plane;
    g.MT = MT;
    g.NT = NT;
    g.KT = KT;
    g.out = (double *)vC;
    g.ldo = nqx;
    g.m_valid = nqx;
    g.n_valid = 2 * nqy;
    g.scale = ldexp(1.0, -14 - 8 * (PD - 1));  // (1/128)^2 per unit of level 0, Horner over PD levels
    g.err = (int *)flags;
    // CTAs that run together work on the same K part of neighbouring output tiles, so they read the same
    // k tiles, which stay in L2.  K is cut into parts so that the last wave of CTAs is nearly full.
    uint32_t ks = 1;
    {
      const uint32_t tiles = MT * NT, sms = (uint32_t)ctx->num_sms;
      double best = 0;
      for (uint32_t c = 1; c <= 8 && c <= KT; c++) {
        const uint32_t n = c * tiles, waves = (n + sms - 1) / sms;
        const double fill = (double)n / ((double)waves * sms);
        if (fill > best + 0.02) {
          best = fill;
          ks = c;
        }
      }
    }
    g.ksplit = ks;
    if ((st = launch_digit_gemm<PlaneScheme, false>(ctx, g, ks * MT * NT))) return st;
    plane_accum_kernel<<<(unsigned)((npix + 255) / 256), 256, 0, ctx->stream>>>(
        (const double *)vC, nqx, nqy, qx0, dqx, qy0, dqy, vcoef ? (const double *)vcoef + 9 * e : nullptr,
        vcoef ? 0.0 : sl[e], Ar, Ai);
    XNS_LAUNCHED(ctx);
  }
  plane_intensity_kernel<<<(unsigned)((npix + 255) / 256), 256, 0, ctx->stream>>>(Ar, Ai, npix, 1.0 / dc.ntot,
                                                                                  (double *)vI);
  XNS_LAUNCHED(ctx);
  if ((st = xns_stage_end(ctx, STAGE_2D))) return st;
  if ((st = xns_timer_stop(ctx))) return st;
  int err = 0;
  XNS_CUDA(ctx, cudaMemcpyAsync(&err, flags, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaMemcpyAsync(I, vI, sizeof(double) * npix, cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (err) return xns_fail(ctx, XNS_ERR_CUDA, "plane: a pipeline wait ran out of time");
  return XNS_OK;
}
