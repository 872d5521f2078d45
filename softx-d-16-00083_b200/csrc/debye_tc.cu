// Exact Debye double sum on the integer tensor cores (tcgen05 kind::i8), for uniform q meshes:
//
//   S_c(q_k) = sum_{pairs of class c} sin(q_k r) / r,   q_k = q0 + k dq
//
// (the pair sum of calcIntDebye / calcIntPartialDebye, CalcFunctions.cpp:576-583 and 698-712; the
// epilogue of the sinc engine applies 1/q, the +1e-8 term, the weights and the self term).
//
// The mesh is split into coarse points Q_a = q_{c_a}, c_a = a (2H + 1) + H, and offsets q_b = b dq,
// |b| <= H, so that sin((Q_a +- q_b) r) = sin(Q_a r) cos(q_b r) +- cos(Q_a r) sin(q_b r).  Per pair
// record r (the K dimension of a GEMM):
//   A (128 rows): sin(Q_a r) for up to 64 coarse points, then cos(Q_a r) (rows of unused points zero);
//   B (32 rows):  cos(q_b r) s(r) for b = 0..15, then sin(q_b r) s(r), s(r) = r_min / r <= 1
//                 (rows of offsets past H are zero);
// C = A B^T summed over records gives C_sc (sin rows x cos columns) and C_cs (cos rows x sin columns),
// and S(Q_a +- q_b) = (C_sc +- C_cs) / r_min.  Both operands are written as 8-bit digits (A:
// round(127 v 2^16) in three, the top one signed; B: round(127 v 2^24) in four signed ones).  The four B digit
// planes lie one after another, which makes them one 128-row operand: one MMA per A digit plane i and
// K step (N = 128, 96, 64: B planes 0 .. 3 - i) multiplies exactly into int32 tensor-memory
// accumulators the nine digit products of level i + j <= 3, and the drain warps combine them by level
// in FP64 every DT_CH units.  Every term is thus carried to ~6e-8 (A) and 2^-31 r / r_min (B) of its size and summed in
// integers, against FP32 rounding per term and FP32 block sums in the sinc engine; the call falls
// back to the sinc engine when r_max / r_min > 2^8.
//
// One CTA per SM, units (a tile pair of 8 x 16 atoms = 128 records, times the q tiles) split evenly
// over the CTAs.  Warp 0 issues the MMAs, warps 1-4 drain tensor memory, warps 5-8 make the records:
// thread k computes record k's FP64 sines and cosines (e^{i Q_0 r}, the coarse and offset steps and
// their powers) for every unit into the record table of the unit's generator group, as soon as the
// group has read its previous unit (the atom coordinates of the next unit load meanwhile).  Warps 9-24 are two generator groups of eight that make the digits of
// alternate units, each group into its own stage: lane l of the group's warp w writes records
// 4l .. 4l + 3 of A rows PA w .. PA w + PA - 1 (and 64 + ...) and B rows 2w, 2w + 1 (and 16 + ...), one
// 32-bit store per (row, digit plane) into the 128-byte-swizzled K-major stage.  Waits are bounded
// (tc_ptx.cuh): record and generator threads each wait on the mbarriers themselves, and the drain warps
// share a named barrier behind a single bounded waiter.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cmath>

#include "schedule.cuh"
#include "sinc_engine.cuh"
#include "tc_ptx.cuh"

using namespace xns_ptx;

namespace {

constexpr int DT_TA = 8, DT_TB = 16;     // atoms of a unit's a-tile and b-tile
constexpr int DT_K = DT_TA * DT_TB;      // 128 records per unit: one 128-byte row per operand row
constexpr int DT_M = 128, DT_QA = 64;    // A rows: sin and cos of 64 coarse points
constexpr int DT_N = 32;                 // B rows: cos and sin of up to 16 offsets
constexpr int DT_NA = 3, DT_NB = 4;              // digits of A and B
constexpr int DT_APL = DT_M * DT_K, DT_BPL = DT_N * DT_K;  // bytes per digit plane
constexpr int DT_STAGE = DT_NA * DT_APL + DT_NB * DT_BPL;  // 64 KB
constexpr int DT_STAGES = 3;   // unit i in stage i % 3: its MMAs run beside the next two units' digits
constexpr int DT_GROUPS = 2;   // generator groups: group i % 2 makes unit i
// Units per accumulator chunk: an accumulator gains one digit product of |.| <= 255 * 128 per record,
// so 256 units (32768 records) keep every int32 sum below 1.07e9.
constexpr int DT_CH = 256;
constexpr int DT_GEN = 8;                                  // warps of a generator group
constexpr int DT_REC = 4;                                  // record warps: one record a thread
constexpr int DT_W_REC = 5, DT_W_GEN = DT_W_REC + DT_REC;  // first record warp, first generator warp
constexpr int DT_THREADS = 32 * (DT_W_GEN + DT_GROUPS * DT_GEN);  // MMA, 4 drain, 4 record, generators
// Accumulators: A digit plane i times B planes 0 .. 3 - i (the products of level i + j <= 3; the others
// are below 2^-32 of a term) at columns 128 i .. (B plane j in columns 32 j ..), one buffer: the MMAs of
// a chunk wait until the previous chunk has been drained.
constexpr uint32_t DT_NB_ROWS = DT_NB * DT_N;              // 128
constexpr uint32_t DT_TMEM_COLS = 512;

// Per-record FP64 values of one unit (e^{i x} as (cos x, sin x)), record k at index (k % 4) 32 + k / 4:
// lane l reads its records 4l .. 4l + 3 as four runs of 32 consecutive entries (no bank conflicts).
// Generator warp w starts at coarse point PA w (E0 WP^w) and offset 2w (F2^w).
struct RecTab {
  double2 E0[DT_K];               // e^{i Q_0 r}: the tile's first coarse point
  double2 W1[DT_K];               // e^{i (2H+1) dq r}: the coarse step
  double2 WP[2][DT_K];            // W1^PA, W1^2PA: steps between generator warps (W1^4PA = WP[1]^2)
  double2 F[3][DT_K];             // e^{i dq r}: the offset step, and its squares F^2, F^4 (F^8 = F[2]^2)
  double s[DT_K];                 // r_min / r, 0 for a record that does not count
};
__device__ __forceinline__ uint32_t rec_slot(uint32_t k) { return (k & 3u) * 32u + (k >> 2); }
// Record tables, one per generator group (unit i in table i % 2), written by the record warps as soon
// as the group has read the table's previous unit.
constexpr int DT_NREC = DT_GROUPS;
constexpr int DT_SMEM = DT_STAGES * DT_STAGE + DT_NREC * (int)sizeof(RecTab) + 1024;
static_assert(DT_SMEM <= 232448, "stages and record tables fit in shared memory");

struct DtArgs {
  const double *X, *Y, *Z;
  const SegPair *sp;
  int nsp;
  unsigned long long ntp;  // this shard's tile pairs: shard + nshard * j, j < ntp
  uint32_t shard, nshard;
  uint32_t MT;             // q tiles (64 coarse points each)
  uint32_t H;              // offsets |b| <= H (H < 16)
  uint32_t PA;             // coarse points per generator warp (8 PA <= 64; A rows past 8 PA are zero)
  double q0, dq;
  uint32_t nq, ncls;
  const unsigned long long *dmin2;  // the closest pair's squared distance (FP64 bits): B scale s = r_min / r
  double *out;             // [grid][ncls][nq], zeroed: each CTA's sums in its own slice
  double *cbuf;            // [grid][128][16]: each CTA's row sums at a segment's end
  double *eps_hist;        // the +1e-8 histogram [ncls][eps_nb] (null: not kept)
  uint32_t eps_nb;
  double eps_inv_bw;
  int *err;
  unsigned long long wait_ns;
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(__fma_rn(a.x, b.x, -a.y * b.y), __fma_rn(a.x, b.y, a.y * b.x));
}

// The record (a pair of atoms) k of a unit: its atoms, its class, and whether it counts.
struct RecLoc {
  uint32_t a, b, cls;
  bool valid;
};
__device__ __forceinline__ RecLoc locate(const DtArgs &g, unsigned long long tp, uint32_t k) {
  int s;
  uint32_t I, J;
  xns_decode_tile(g.sp, g.nsp, tp, &s, &I, &J);
  const SegPair p = g.sp[s];
  const uint32_t ib = I * DT_TA, jb = J * DT_TB, ii = k / DT_TB, jj = k % DT_TB;
  // a "same" entry may name an a-tile past the segment's end (schedule.cuh): it is empty
  const uint32_t ni = ib < p.na ? min((uint32_t)DT_TA, p.na - ib) : 0u, nj = min((uint32_t)DT_TB, p.nb - jb);
  RecLoc L;
  L.cls = p.cls;
  L.valid = !(ii >= ni || jj >= nj || (p.same && ib + ii >= jb + jj));
  L.a = L.valid ? p.a0 + ib + ii : 0u;
  L.b = L.valid ? p.b0 + jb + jj : 0u;
  return L;
}
__device__ __forceinline__ uint32_t unit_class(const DtArgs &g, unsigned long long u) {
  int s;
  uint32_t I, J;
  xns_decode_tile(g.sp, g.nsp, g.shard + (unsigned long long)g.nshard * (u % g.ntp), &s, &I, &J);
  return g.sp[s].cls;
}
// (q tile, class) of unit u: an accumulator chunk never spans two of them
__device__ __forceinline__ unsigned long long unit_key(const DtArgs &g, unsigned long long u) {
  return (u / g.ntp) << 32 | unit_class(g, u);
}

// Base-256 digits of N = round(127 v 2^16) (A, three) and round(127 v 2^24) (B, four), |v| <= 1: the
// integer lands in the low word of an FMA with 1.5 * 2^52.  A: the bytes of that word as they are,
// N = d0 2^16 + d1 2^8 + d2 with d0 = floor(N / 2^16) signed (|d0| <= 127) and d1, d2 unsigned (the A
// planes are separate MMAs, each with its own signedness).  B: adding 0x808080 carries a bias of 128
// into every byte, and flipping the bias bits back leaves signed digits in [-128, 127] as bytes, the
// most significant highest (B's four planes are one operand: one signedness).
__device__ __forceinline__ uint32_t digits_a(double v) {
  return (uint32_t)__double2loint(__fma_rn(v, 127.0 * 65536.0, 6755399441055744.0));
}
__device__ __forceinline__ uint32_t digits_b(double v) {
  const uint32_t lo = (uint32_t)__double2loint(__fma_rn(v, 127.0 * 16777216.0, 6755399441055744.0));
  return (lo + 0x808080u) ^ 0x808080u;
}

__device__ __forceinline__ uint32_t chunk_off(uint32_t row, uint32_t ch) {
  return (row >> 3) * 1024u + (row & 7u) * 128u + (((ch ^ row) & 7u) << 4);
}

__device__ __forceinline__ void tc_mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
      : "memory");
}

__global__ void __launch_bounds__(DT_THREADS, 1) debye_tc_kernel(const DtArgs g) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) unsigned long long bars[2 * DT_STAGES + 5 + 2 * DT_NREC];
  __shared__ uint32_t tmem_sh;
  __shared__ int abort_sh, drain_stop;
  const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
  uint8_t *gsm = smem_raw + (base - smem_u32(smem_raw));
  RecTab *rec = reinterpret_cast<RecTab *>(gsm + DT_STAGES * DT_STAGE);
  const uint32_t full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[DT_STAGES]);
  const uint32_t tfull0 = smem_u32(&bars[2 * DT_STAGES]), tempty0 = smem_u32(&bars[2 * DT_STAGES + 2]);
  const uint32_t drain = smem_u32(&bars[2 * DT_STAGES + 4]);
  // record table b: rfull0 + 8 b (written), rempty0 + 8 b (read by its generator group)
  const uint32_t rfull0 = smem_u32(&bars[2 * DT_STAGES + 5]), rempty0 = rfull0 + 8 * DT_NREC;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  volatile int *abort = &abort_sh;

  if (threadIdx.x == 0) {
    for (int s = 0; s < DT_STAGES; s++) {
      mbar_init(full0 + 8 * s, 32 * DT_GEN);  // every thread of the stage's generator group
      mbar_init(empty0 + 8 * s, 1);           // the MMAs' commit
    }
    mbar_init(tfull0, 1);       // the chunk's MMAs
    mbar_init(tempty0, 128);    // the drain warps
    mbar_init(drain, 1);
    for (int b = 0; b < DT_NREC; b++) {
      mbar_init(rfull0 + 8 * b, 32 * DT_REC);   // every record thread
      mbar_init(rempty0 + 8 * b, 32 * DT_GEN);  // every thread of the consuming generator group
    }
    abort_sh = 0;
    drain_stop = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_sh)),
                 "r"(DT_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_sh;
  // r_min from the closest-pair pass (read on the device: no round trip through the host); one unit of
  // the level sum (levels i + j <= 3, N_A N_B / 2^16) with A = N_A / (127 2^16), B = N_B / (127 2^24)
  // and S = sum A B / r_min
  double rmin;
  {
    const double m2 = __longlong_as_double((long long)*g.dmin2);
    rmin = (m2 > 0.0 && m2 < INFINITY) ? sqrt(m2) * (1.0 - 1e-12) : 1.0;
  }
  const double unit = 1.0 / (127.0 * 127.0 * 16777216.0 * rmin);
  const unsigned long long units = g.ntp * g.MT;
  const unsigned long long u0 = units * blockIdx.x / gridDim.x, u1 = units * (blockIdx.x + 1) / gridDim.x;

  if (warp == 0) {
    if (lane == 0) {  // MMA issuer
      // kind::i8: S32 accumulator (2), A signed (1, the top digit plane) or unsigned (0), B signed (1),
      // K-major, M = 128, N = 32 (4 - i) for A plane i: B planes 0 .. 3 - i
      uint32_t idesc[DT_NA];
#pragma unroll
      for (int di = 0; di < DT_NA; di++)
        idesc[di] = (2u << 4) | (di == 0 ? 1u << 7 : 0u) | (1u << 10) | ((uint32_t)(DT_N * (DT_NB - di) >> 3) << 17) |
                    ((uint32_t)(DT_M >> 4) << 24);
      uint32_t chunk = 0, in_chunk = 0;
      bool issued = false;
      unsigned long long i = 0, key = u0 < u1 ? unit_key(g, u0) : 0;
      for (unsigned long long u = u0; u < u1; ++u, ++i) {
        const uint32_t s = (uint32_t)(i % DT_STAGES), k = (uint32_t)(i / DT_STAGES);
        const unsigned long long nkey = u + 1 < u1 ? unit_key(g, u + 1) : ~0ull;
        const bool last = nkey != key || in_chunk + 1 == DT_CH;
        if (in_chunk == 0 && chunk >= 1) {  // the drain warps have read the previous chunk
          if (!mbar_wait(tempty0, (chunk - 1) & 1u, abort, g.wait_ns)) {
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
        const uint32_t a0 = base + s * DT_STAGE, b0 = a0 + DT_NA * DT_APL;
#pragma unroll
        for (int ks = 0; ks < DT_K / 32; ks++) {  // K = 32 int8 (32 bytes) per instruction
          const uint32_t off = ks * 32;
          const uint32_t acc = (in_chunk == 0 && ks == 0) ? 0u : 1u;  // a chunk's first unit overwrites
#pragma unroll
          for (int di = 0; di < DT_NA; di++)
            tc_mma_i8(tmem + di * DT_NB_ROWS, sw128_desc(a0 + di * DT_APL + off), sw128_desc(b0 + off), idesc[di], acc);
        }
        issued = true;
        tc_commit(empty0 + 8 * s);
        in_chunk++;
        if (last) {
          tc_commit(tfull0);
          chunk++;
          in_chunk = 0;
        }
        key = nkey;
      }
      if (*abort && issued) {
        tc_commit(drain);
        mbar_wait(drain, 0, nullptr, DRAIN_LIMIT_NS);
      }
    }
  } else if (warp <= 4) {
    // drain: warp w reads TMEM lanes 32 (w % 4) .. + 31 (rows), every chunk.  Sin rows (0-63) need the
    // cos columns (0-15), cos rows (64-127) the sin columns (16-31).
    const uint32_t wq = warp & 3;
    const uint32_t row = wq * 32 + lane, colb = wq >= 2 ? 16u : 0u;
    const uint32_t lane_addr = tmem + ((wq * 32u) << 16) + colb;
    double sum[16];
#pragma unroll
    for (int j = 0; j < 16; j++) sum[j] = 0.0;
    uint32_t chunk = 0, in_chunk = 0;
    unsigned long long key = u0 < u1 ? unit_key(g, u0) : 0;
    for (unsigned long long u = u0; u < u1; ++u) {
      const unsigned long long nkey = u + 1 < u1 ? unit_key(g, u + 1) : ~0ull;
      const bool seg_end = nkey != key;
      const bool last = seg_end || in_chunk + 1 == DT_CH;
      in_chunk++;
      if (last) {
        in_chunk = 0;
        {
          // one bounded wait for the chunk, then the drain warps' barrier (the stop flag is read after it)
          if (row == 32) {  // warp 1, lane 0
            if (!mbar_wait(tfull0, chunk & 1u, abort, g.wait_ns)) {
              abort_sh = 1;
              atomicOr(g.err, 1);
              drain_stop = 1;
            }
          }
          asm volatile("bar.sync 4, 128;" ::: "memory");
          if (drain_stop) break;
          tc_fence_after();
#pragma unroll
          for (int hf = 0; hf < 2; hf++) {  // 8 columns at a time
            double t[8];
#pragma unroll
            for (int j = 0; j < 8; j++) t[j] = 0.0;
#pragma unroll
            for (int lev = 0; lev < DT_NB; lev++) {  // Horner over the levels i + j <= 3, top first
#pragma unroll
              for (int j = 0; j < 8; j++) t[j] *= 256.0;
#pragma unroll
              for (int di = 0; di < DT_NA; di++) {
                const int ej = lev - di;
                if (ej < 0 || ej >= DT_NB - di) continue;  // the products the MMAs keep
                uint32_t rr[8];
                tc_ld8_raw(lane_addr + di * DT_NB_ROWS + ej * DT_N + 8 * hf, rr);
#pragma unroll
                for (int j = 0; j < 8; j++) t[j] += (double)(int)rr[j];
              }
            }
#pragma unroll
            for (int j = 0; j < 8; j++) sum[8 * hf + j] += t[j];
          }
          tc_fence_before();
          mbar_arrive(tempty0);
        }
        chunk++;
        if (seg_end) {
          // the sums of the (q tile, class) segment into this CTA's slice, in a fixed order (no atomics:
          // the result does not depend on timing): the rows' sums go to this CTA's scratch, then
          // q = Q_a + b dq (a = k / (2H + 1), |b| <= H) gets C_sc[a][|b|] + sign(b) C_cs[a][|b|]
          const uint32_t mt = (uint32_t)(key >> 32), cls = (uint32_t)key, span = 2 * g.H + 1;
          double *cb = g.cbuf + (size_t)blockIdx.x * DT_M * 16;
#pragma unroll
          for (int j = 0; j < 16; j++) {
            cb[row * 16 + j] = sum[j];
            sum[j] = 0.0;
          }
          asm volatile("bar.sync 4, 128;" ::: "memory");
          double *o = g.out + ((size_t)blockIdx.x * g.ncls + cls) * g.nq;
          const uint32_t k0 = mt * DT_QA * span, k1 = min(g.nq, k0 + DT_QA * span);
          for (uint32_t k = k0 + row; k < k1; k += DT_M) {
            const uint32_t a = (k - k0) / span;
            const int b = (int)((k - k0) % span) - (int)g.H, bb = b < 0 ? -b : b;
            const double csc = cb[a * 16 + bb], ccs = cb[(DT_QA + a) * 16 + bb];
            o[k] += (csc + (b < 0 ? -ccs : ccs)) * unit;
          }
          asm volatile("bar.sync 4, 128;" ::: "memory");  // before the next segment rewrites the scratch
        }
      }
      key = nkey;
    }
  } else if (warp < DT_W_GEN) {
    // record warps: thread kr makes record kr of every unit of this CTA (unit i into table i % DT_NREC)
    const uint32_t kr = threadIdx.x - DT_W_REC * 32, ks = rec_slot(kr);
    const double dqA = (2.0 * g.H + 1.0) * g.dq;
    // the record of the first unit: located and its coordinates loaded
    RecLoc loc{0, 0, 0, false};
    double ca[3] = {0, 0, 0}, cb[3] = {0, 0, 0};
    if (u0 < u1) {
      loc = locate(g, g.shard + (unsigned long long)g.nshard * (u0 % g.ntp), kr);
      if (loc.valid) {
        ca[0] = g.X[loc.a], ca[1] = g.Y[loc.a], ca[2] = g.Z[loc.a];
        cb[0] = g.X[loc.b], cb[1] = g.Y[loc.b], cb[2] = g.Z[loc.b];
      }
    }
    uint32_t i = 0;
    for (unsigned long long u = u0; u < u1; ++u, ++i) {
      const uint32_t b = i % DT_NREC, p = i / DT_NREC, mt = (uint32_t)(u / g.ntp);
      double r = 0.0;
      if (loc.valid) {
        const double dx = ca[0] - cb[0], dy = ca[1] - cb[1], dz = ca[2] - cb[2];
        r = sqrt(dx * dx + dy * dy + dz * dz);
      }
      const uint32_t cls = loc.cls;
      if (u + 1 < u1) {  // the next unit's record: its loads run during this unit's work
        loc = locate(g, g.shard + (unsigned long long)g.nshard * ((u + 1) % g.ntp), kr);
        if (loc.valid) {
          ca[0] = g.X[loc.a], ca[1] = g.Y[loc.a], ca[2] = g.Z[loc.a];
          cb[0] = g.X[loc.b], cb[1] = g.Y[loc.b], cb[2] = g.Z[loc.b];
        }
      }
      // the record's values, in registers while the table may still be read
      double sn, cs;
      const double Q0 = g.q0 + ((double)mt * DT_QA * (2.0 * g.H + 1.0) + g.H) * g.dq;
      xns_math::xns_sincos64(Q0 * r, &sn, &cs);
      const double2 e0 = make_double2(cs, sn);
      xns_math::xns_sincos64(dqA * r, &sn, &cs);
      const double2 w1 = make_double2(cs, sn);
      double2 wp = make_double2(1.0, 0.0), bp = w1;  // w1^PA by squaring
      for (uint32_t e = g.PA; e; e >>= 1) {
        if (e & 1u) wp = cmul(wp, bp);
        bp = cmul(bp, bp);
      }
      const double2 wp2 = cmul(wp, wp);
      xns_math::xns_sincos64(g.dq * r, &sn, &cs);
      const double2 f1 = make_double2(cs, sn), f2 = cmul(f1, f1), f4 = cmul(f2, f2);
      const bool valid = r > 0.0;
      const double ir = valid ? 1.0 / r : 0.0;
      if (valid && mt == 0 && g.eps_hist) {
        const uint32_t kb = (uint32_t)fmin(r * g.eps_inv_bw, (double)(g.eps_nb - 1));
        atomicAdd(g.eps_hist + (size_t)cls * g.eps_nb + kb, ir * ir);
      }
      // wait (bounded) until the generator group has read the table's previous unit
      bool ok = !*abort;
      if (ok && p > 0) ok = mbar_wait(rempty0 + 8 * b, (p - 1) & 1u, abort, g.wait_ns);
      if (!ok) {
        abort_sh = 1;
        atomicOr(g.err, 1);
        break;
      }
      RecTab &R = rec[b];
      R.E0[ks] = e0;
      R.W1[ks] = w1;
      R.WP[0][ks] = wp;
      R.WP[1][ks] = wp2;
      R.F[0][ks] = f1;
      R.F[1][ks] = f2;
      R.F[2][ks] = f4;
      R.s[ks] = rmin * ir;
      mbar_arrive(rfull0 + 8 * b);
    }
  } else {
    // generators: group G makes the units i with i % 2 == G (i counted from u0), unit i into stage i % 3
    const uint32_t G = (uint32_t)(warp - DT_W_GEN) / DT_GEN, t = threadIdx.x - (DT_W_GEN + G * DT_GEN) * 32, gw = t >> 5;
    // B rows of offsets past H and A rows of coarse points past 8 PA (sin rows a, cos rows 64 + a) stay
    // zero: group G clears them once in the stages s with s % 2 == G (before its first arrival on any
    // stage's full barrier; a row is 128 contiguous bytes, whatever the swizzle order of its chunks)
    for (uint32_t sz = G; sz < (uint32_t)DT_STAGES; sz += DT_GROUPS) {
      for (uint32_t e = t; e < (uint32_t)DT_NB * DT_N * 32u; e += 32 * DT_GEN) {
        const uint32_t pl = e / (DT_N * 32u), r = (e / 32u) % DT_N, w4 = e % 32u;
        if ((r & 15u) > g.H) *(uint32_t *)(gsm + sz * DT_STAGE + DT_NA * DT_APL + pl * DT_BPL + r * 128u + w4 * 4u) = 0u;
      }
      for (uint32_t e = t; e < (uint32_t)DT_NA * DT_M * 32u; e += 32 * DT_GEN) {
        const uint32_t pl = e / (DT_M * 32u), r = (e / 32u) % DT_M, w4 = e % 32u;
        if ((r & 63u) >= DT_GEN * g.PA) *(uint32_t *)(gsm + sz * DT_STAGE + pl * DT_APL + r * 128u + w4 * 4u) = 0u;
      }
    }
    const uint32_t l = lane, ch = l >> 2, bo = 4u * (l & 3u);
    for (unsigned long long u = u0 + G, iu = G; u < u1; u += DT_GROUPS, iu += DT_GROUPS) {
      const uint32_t b = (uint32_t)(iu % DT_NREC), p = (uint32_t)(iu / DT_NREC);
      const uint32_t s = (uint32_t)(iu % DT_STAGES), k = (uint32_t)(iu / DT_STAGES);  // stage, its use
      // every thread waits (bounded) for the stage and the unit's record table itself: the group's warps
      // run ahead of one another as far as the stages allow, and a wait that runs out stops them all
      bool ok = !*abort;
      if (ok && k > 0) ok = mbar_wait(empty0 + 8 * s, (k - 1) & 1u, abort, g.wait_ns);
      if (ok) ok = mbar_wait(rfull0 + 8 * b, p & 1u, abort, g.wait_ns);
      if (!ok) {
        abort_sh = 1;
        atomicOr(g.err, 1);
        break;
      }
      const RecTab &R = rec[b];
      uint8_t *st = gsm + s * DT_STAGE;
      // A: rows 8 gw + a (sin) and 64 + 8 gw + a (cos), records 4 l + c
      {
        double2 z[4], w1[4];
#pragma unroll
        for (int c = 0; c < 4; c++) {  // coarse point PA gw: E0 WP^gw
          const uint32_t kc = c * 32 + l;
          z[c] = R.E0[kc];
          w1[c] = R.W1[kc];
          if (gw & 1u) z[c] = cmul(z[c], R.WP[0][kc]);
          if (gw & 2u) z[c] = cmul(z[c], R.WP[1][kc]);
          if (gw & 4u) z[c] = cmul(z[c], cmul(R.WP[1][kc], R.WP[1][kc]));
        }
#pragma unroll 2
        for (uint32_t a = 0; a < g.PA; a++) {
          uint32_t ds[4], dc[4];
#pragma unroll
          for (int c = 0; c < 4; c++) {
            ds[c] = digits_a(z[c].y);
            dc[c] = digits_a(z[c].x);
            z[c] = cmul(z[c], w1[c]);
          }
          const uint32_t m = g.PA * gw + a, off = chunk_off(m, ch) + bo;  // cos row m + 64: + 8192
          // planes: digit 0 (most significant) = byte 2
          const uint32_t s01 = __byte_perm(ds[0], ds[1], 0x5140), s23 = __byte_perm(ds[2], ds[3], 0x5140);
          const uint32_t s2a = __byte_perm(ds[0], ds[1], 0x0062), s2b = __byte_perm(ds[2], ds[3], 0x0062);
          const uint32_t c01 = __byte_perm(dc[0], dc[1], 0x5140), c23 = __byte_perm(dc[2], dc[3], 0x5140);
          const uint32_t c2a = __byte_perm(dc[0], dc[1], 0x0062), c2b = __byte_perm(dc[2], dc[3], 0x0062);
          *(uint32_t *)(st + off) = __byte_perm(s2a, s2b, 0x5410);
          *(uint32_t *)(st + DT_APL + off) = __byte_perm(s01, s23, 0x7632);
          *(uint32_t *)(st + 2 * DT_APL + off) = __byte_perm(s01, s23, 0x5410);
          *(uint32_t *)(st + off + 8192) = __byte_perm(c2a, c2b, 0x5410);
          *(uint32_t *)(st + DT_APL + off + 8192) = __byte_perm(c01, c23, 0x7632);
          *(uint32_t *)(st + 2 * DT_APL + off + 8192) = __byte_perm(c01, c23, 0x5410);
        }
      }
      // B: rows b = 2 gw + e (cos) and 16 + b (sin), b <= H
      if (2 * gw <= g.H) {
        double2 z[4], f1[4];
        double sc[4];
#pragma unroll
        for (int c = 0; c < 4; c++) {  // offset 2 gw: F^(2 gw)
          const uint32_t kc = c * 32 + l;
          z[c] = (gw & 1u) ? R.F[1][kc] : make_double2(1.0, 0.0);
          if (gw & 2u) z[c] = cmul(z[c], R.F[2][kc]);
          if (gw & 4u) z[c] = cmul(z[c], cmul(R.F[2][kc], R.F[2][kc]));
          f1[c] = R.F[0][kc];
          sc[c] = R.s[kc];
        }
        uint8_t *bst = st + DT_NA * DT_APL;
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const uint32_t b = 2 * gw + e;
          if (b > g.H) break;
          uint32_t dcs[4], dsn[4];
#pragma unroll
          for (int c = 0; c < 4; c++) {
            dcs[c] = digits_b(z[c].x * sc[c]);
            dsn[c] = digits_b(z[c].y * sc[c]);
            z[c] = cmul(z[c], f1[c]);
          }
          const uint32_t offc = chunk_off(b, ch) + bo, offs = chunk_off(16 + b, ch) + bo;
          // planes: digit 0 (most significant) = byte 3
          {
            const uint32_t x01 = __byte_perm(dcs[0], dcs[1], 0x5140), x23 = __byte_perm(dcs[2], dcs[3], 0x5140);
            const uint32_t y01 = __byte_perm(dcs[0], dcs[1], 0x7362), y23 = __byte_perm(dcs[2], dcs[3], 0x7362);
            *(uint32_t *)(bst + offc) = __byte_perm(y01, y23, 0x7632);
            *(uint32_t *)(bst + DT_BPL + offc) = __byte_perm(y01, y23, 0x5410);
            *(uint32_t *)(bst + 2 * DT_BPL + offc) = __byte_perm(x01, x23, 0x7632);
            *(uint32_t *)(bst + 3 * DT_BPL + offc) = __byte_perm(x01, x23, 0x5410);
          }
          {
            const uint32_t x01 = __byte_perm(dsn[0], dsn[1], 0x5140), x23 = __byte_perm(dsn[2], dsn[3], 0x5140);
            const uint32_t y01 = __byte_perm(dsn[0], dsn[1], 0x7362), y23 = __byte_perm(dsn[2], dsn[3], 0x7362);
            *(uint32_t *)(bst + offs) = __byte_perm(y01, y23, 0x7632);
            *(uint32_t *)(bst + DT_BPL + offs) = __byte_perm(y01, y23, 0x5410);
            *(uint32_t *)(bst + 2 * DT_BPL + offs) = __byte_perm(x01, x23, 0x7632);
            *(uint32_t *)(bst + 3 * DT_BPL + offs) = __byte_perm(x01, x23, 0x5410);
          }
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes -> tensor-core reads
      mbar_arrive(full0 + 8 * s);
      mbar_arrive(rempty0 + 8 * b);  // this thread is done with the record table
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(DT_TMEM_COLS) : "memory");
}

// The smallest nonzero pair distance squared (as FP64 bits, for atomicMin) over this shard's units: a
// warp per unit, lane l its records 4l .. 4l + 3 (one a-atom, four b-atoms).
__global__ void debye_tc_rmin_kernel(const DtArgs g, unsigned long long *dmin) {
  double m = INFINITY;
  const uint32_t lane = threadIdx.x & 31, ii = lane >> 2, jj0 = 4 * (lane & 3);
  const unsigned long long nw = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
  for (unsigned long long w = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < g.ntp; w += nw) {
    int s;
    uint32_t I, J;
    xns_decode_tile(g.sp, g.nsp, g.shard + (unsigned long long)g.nshard * w, &s, &I, &J);
    const SegPair p = g.sp[s];
    const uint32_t ib = I * DT_TA, jb = J * DT_TB;
    const uint32_t ni = ib < p.na ? min((uint32_t)DT_TA, p.na - ib) : 0u, nj = min((uint32_t)DT_TB, p.nb - jb);
    if (ii >= ni) continue;
    const uint32_t a = p.a0 + ib + ii;
    const double xa = g.X[a], ya = g.Y[a], za = g.Z[a];
#pragma unroll
    for (uint32_t c = 0; c < 4; c++) {
      const uint32_t jj = jj0 + c;
      if (jj >= nj || (p.same && ib + ii >= jb + jj)) continue;
      const uint32_t b = p.b0 + jb + jj;
      const double dx = xa - g.X[b], dy = ya - g.Y[b], dz = za - g.Z[b];
      const double d2 = dx * dx + dy * dy + dz * dz;  // the kernel's r is the square root of this sum
      if (d2 > 0.0) m = fmin(m, d2);
    }
  }
  for (int o = 16; o; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0 && m < INFINITY) atomicMin(dmin, (unsigned long long)__double_as_longlong(m));
}

// Adds the slices 1 .. grid - 1 of p ([grid][n]) to slice 0 in a fixed order: warp w of a block sums
// the slices 1 + w, 9 + w, ... of 32 consecutive entries, then the block adds the warps' sums in order.
__global__ void __launch_bounds__(256) slice_sum_kernel(double *__restrict__ p, uint32_t grid, size_t n) {
  __shared__ double part[8][32];
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const size_t i = (size_t)blockIdx.x * 32 + lane;
  double s = 0.0;
  if (i < n)
    for (uint32_t c = 1 + w; c < grid; c += 8) s += p[(size_t)c * n + i];
  part[w][lane] = s;
  __syncthreads();
  if (w == 0 && i < n) {
    double t = p[i];
#pragma unroll
    for (int k = 0; k < 8; k++) t += part[k][lane];
    p[i] = t;
  }
}

}  // namespace

namespace xns_sinc {

int debye_tc(xns_ctx *ctx, const DevCoords &dc, const std::vector<Segment> &sa, const std::vector<Segment> &sb,
             const std::vector<uint32_t> &cls, const std::vector<uint32_t> &same, uint32_t ncls, double q0, double dq,
             uint32_t nq, double rmax, uint32_t shard, uint32_t nshard, bool *used, int *grid_out) {
  *used = false;
  if (nq < 2 || !(dq > 0) || !(rmax > 0)) return XNS_OK;
  std::vector<SegPair> sched;
  const unsigned long long ntp_all = xns_build_schedule(sa, sb, cls, same, DT_TA, DT_TB, &sched);
  const unsigned long long ntp = ntp_all > shard ? (ntp_all - shard + nshard - 1) / nshard : 0;
  // offsets |b| <= H around 64 coarse points per q tile
  // offsets |b| <= H and coarse points per generator warp PA: the fewest values per record (2 per
  // coarse point made, 2 per offset) whose coarse points cover the mesh; past 64 (2H + 1) points, q
  // tiles of 64 coarse points and H = 15
  uint32_t H = 15, PA = DT_QA / DT_GEN, MT = 1;
  if (nq > (uint32_t)DT_QA * 31u) {
    MT = (nq + DT_QA * 31u - 1) / (DT_QA * 31u);
  } else {
    uint32_t best = ~0u;
    for (uint32_t h = 1; h <= 15; h++) {
      const uint32_t na = (nq + 2 * h) / (2 * h + 1), pa = (na + DT_GEN - 1) / DT_GEN;
      if (pa > DT_QA / DT_GEN) continue;
      const uint32_t cost = 2 * DT_GEN * pa + 2 * (h + 1);
      if (cost < best) best = cost, H = h, PA = pa;
    }
  }
  SegPair *d_sp = nullptr;
  int st;
  if (ntp && (st = xns_upload_schedule(ctx, sched, &d_sp))) return st;
  DtArgs g{};
  g.X = dc.x;
  g.Y = dc.y;
  g.Z = dc.z;
  g.sp = d_sp;
  g.nsp = (int)sched.size();
  g.ntp = ntp;
  g.shard = shard;
  g.nshard = nshard;
  g.MT = MT;
  g.H = H;
  g.PA = PA;
  g.q0 = q0;
  g.dq = dq;
  g.nq = nq;
  g.ncls = ncls;
  // the smallest distance of the whole structure (every shard) sets the B scale: every shard then writes
  // each term with the same digits, and the shards add up to the one-call sums.  The kernel reads it on
  // the device; the host checks it once the work is queued (a structure with r_max > 256 r_min, where B
  // would lose more than 8 bits, then takes the sinc engine instead)
  void *df;
  if ((st = xns_scratch(ctx, SLOT_FLAGS, 64, &df))) return st;
  unsigned long long *d_min = (unsigned long long *)df;
  int *d_err = (int *)((char *)df + 16);
  XNS_CUDA(ctx, cudaMemsetAsync(d_min, 0x7f, sizeof(unsigned long long), ctx->stream));
  XNS_CUDA(ctx, cudaMemsetAsync(d_err, 0, sizeof(int), ctx->stream));
  if (ntp) {
    DtArgs ga = g;
    ga.shard = 0;
    ga.nshard = 1;
    ga.ntp = ntp_all;
    debye_tc_rmin_kernel<<<ctx->num_sms * 16, 256, 0, ctx->stream>>>(ga, d_min);
    XNS_LAUNCHED(ctx);
  }
  g.dmin2 = d_min;
  g.err = d_err;
  // one CTA per SM; each CTA's sums in its own slice (summed in order by the epilogue), then its scratch
  const unsigned long long units = ntp * MT;
  const unsigned grid = (unsigned)std::max<unsigned long long>(1, std::min<unsigned long long>((unsigned long long)ctx->num_sms, units));
  void *d;
  const size_t ob = sizeof(double) * (size_t)grid * ncls * nq, cbb = sizeof(double) * (size_t)grid * DT_M * 16;
  if ((st = xns_scratch(ctx, SLOT_PARTIAL, ob + cbb, &d))) return st;
  XNS_CUDA(ctx, cudaMemsetAsync(d, 0, ob, ctx->stream));
  g.out = (double *)d;
  g.cbuf = (double *)((char *)d + ob);
  double ebin = 0;
  uint32_t enb = 0;
  eps_layout(rmax, EPS_NB_MAX, &enb, &ebin);
  g.eps_nb = enb;
  g.eps_inv_bw = 1.0 / ebin;
  const size_t hb = sizeof(double) * ncls * enb;
  if ((st = xns_scratch(ctx, SLOT_EPS_HIST, hb, &d))) return st;
  XNS_CUDA(ctx, cudaMemsetAsync(d, 0, hb, ctx->stream));
  g.eps_hist = (double *)d;
  g.wait_ns = WAIT_LIMIT_NS;
  if (ntp) {
    static bool attr_set[XNS_MAX_DEVICES] = {};
    if (ctx->device < 0 || ctx->device >= XNS_MAX_DEVICES || !attr_set[ctx->device]) {
      XNS_CUDA(ctx, cudaFuncSetAttribute(debye_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, DT_SMEM));
      if (ctx->device >= 0 && ctx->device < XNS_MAX_DEVICES) attr_set[ctx->device] = true;
    }
    debye_tc_kernel<<<grid, DT_THREADS, DT_SMEM, ctx->stream>>>(g);
    XNS_LAUNCHED(ctx);
  }
  // the +1e-8 sums from the distance histogram
  const size_t tb = sizeof(double) * ncls * nq;
  if ((st = xns_scratch(ctx, SLOT_EPS_T, tb, &d))) return st;
  XNS_CUDA(ctx, cudaMemsetAsync(d, 0, tb, ctx->stream));
  dim3 eg((nq + 127) / 128, (enb + EPS_RUN - 1) / EPS_RUN, ncls);
  sinc_eps_kernel<<<eg, 128, 0, ctx->stream>>>(g.eps_hist, enb, ebin, q0, dq, nullptr, nq, (double *)d);
  XNS_LAUNCHED(ctx);
  // the CTAs' slices into slice 0, in a fixed order
  if (grid > 1) {
    const size_t n = (size_t)ncls * nq;
    slice_sum_kernel<<<(unsigned)((n + 31) / 32), 256, 0, ctx->stream>>>(g.out, grid, n);
    XNS_LAUNCHED(ctx);
  }
  int herr = 0;
  unsigned long long h_min = 0;
  XNS_CUDA(ctx, cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaMemcpyAsync(&h_min, d_min, sizeof(h_min), cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (herr) return xns_fail(ctx, XNS_ERR_CUDA, "Debye: a tensor-core pipeline wait ran out");
  if (ntp) {
    double m2;
    memcpy(&m2, &h_min, sizeof m2);
    if (!(m2 > 0) || !std::isfinite(m2)) return XNS_OK;          // no pair counts: the sinc engine's path
    if (rmax > 256.0 * sqrt(m2) * (1.0 - 1e-12)) return XNS_OK;  // B would lose more than 8 bits
  }
  *grid_out = 1;
  *used = true;
  return XNS_OK;
}

}  // namespace xns_sinc
