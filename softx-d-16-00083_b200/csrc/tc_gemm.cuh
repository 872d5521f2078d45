// Split-BF16 sinc transform on the 5th-generation tensor cores (tcgen05, TMEM accumulators).
//
//   G[c][q] = sum_k n_c[k] * sin(q r_k) / (q r_k),   r_k = (k + 0.5) * bin
//
// is the histogram -> I(q) contraction of calcInt1DHist (CalcFunctions.cpp:810-911) for many
// histogram columns c at once (structures x element pairs): a dense (q x k) sinc matrix S times a
// (k x c) count matrix H.  Both operands are split into BF16 hi + lo parts (x = hi + lo, |lo| <=
// 2^-9 |x|), and three products Sh*Hh + Sh*Hl + Sl*Hh are accumulated in FP32 in tensor memory; the
// dropped Sl*Hl term is below 2^-16 relative.  K is split over CTAs (stream-K) and the FP32 tile
// sums are added into an FP64 output, so each FP32 accumulator holds at most one CTA's K range.
//
// Operands live in HBM already in the shared-memory image the MMA reads (K-major, 128-byte
// swizzle, 8-row groups of 1024 bytes), so one untiled bulk copy (cp.async.bulk) moves a whole
// tile and no tensor map is needed.
#pragma once
#include <cuda_bf16.h>

#include "xns_internal.cuh"

namespace xns_tc {

constexpr int BM = 128;                            // q rows per tile (MMA M)
constexpr int BK = 64;                             // k per tile: one 128-byte swizzle row of BF16
constexpr int BN_MAX = 256;                        // columns per tile (MMA N), a multiple of 16
constexpr int A_TILE = BM * BK * 2;                // 16 KB
constexpr int B_TILE_MAX = BN_MAX * BK * 2;        // 32 KB
constexpr int STAGES = 2;
constexpr int STAGE_BYTES = 2 * A_TILE + 2 * B_TILE_MAX;
constexpr int THREADS = 192;                       // warp 0 loads, warp 1 issues MMAs, warps 2-5 drain TMEM
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024;
constexpr uint32_t TMEM_COLS = 256;

// Byte offset of element (row, k) of a K-major 128-byte-swizzled tile: rows are 128 bytes, 8 rows
// form a 1024-byte group, and the 16-byte chunk index is XORed with the row's index in its group.
__host__ __device__ inline uint32_t sw128_offset(uint32_t row, uint32_t k) {
  return (row >> 3) * 1024u + (row & 7u) * 128u + ((((k >> 3) ^ row) & 7u) << 4) + (k & 7u) * 2u;
}

struct GemmArgs {
  const uint8_t *Ah, *Al;  // sinc matrix planes: tiles [mt][kt] of A_TILE bytes
  const uint8_t *Bh, *Bl;  // count planes: tiles [nt][kt] of BN*128 bytes
  uint32_t MT, NT, KT, BN;
  double *out;             // out[n * ldo + m], accumulated with FP64 atomics (zeroed by the caller)
  uint32_t ldo, m_valid, n_valid;
  int *err;                // set non-zero when a wait ran out of time
};

}  // namespace xns_tc

// Pack the sinc matrix S[m][k] = sin(q_m r_k)/(q_m r_k) into hi/lo tile planes (MT x KT tiles).
// Rows m >= nq and columns k >= nh are zero.
int xns_tc_pack_sinc(xns_ctx *ctx, const double *d_q, uint32_t nq, double bin, uint32_t nh, uint32_t MT, uint32_t KT,
                     uint8_t *Ah, uint8_t *Al);
// Pack u64 count columns (column c at d_hist + c*ldh, nh bins) into hi/lo tile planes (NT x KT tiles
// of BN rows).
int xns_tc_pack_counts(xns_ctx *ctx, const unsigned long long *d_hist, uint32_t ncols, uint32_t nh, size_t ldh,
                       uint32_t BN, uint32_t NT, uint32_t KT, uint8_t *Bh, uint8_t *Bl);
// out[c*nq + m] = sum_k counts * sinc on the tensor cores (out zeroed here).  grid = 0: one CTA per SM.
int xns_tc_sinc_gemm(xns_ctx *ctx, const xns_tc::GemmArgs &g, int grid);
// Whole transform for ncols device histogram columns: packs (the sinc planes are cached in the
// context for the last q mesh / bin / extent) and multiplies.  d_G receives ncols x nq FP64.
int xns_tc_hist_transform(xns_ctx *ctx, const unsigned long long *d_hist, uint32_t ncols, uint32_t nh, size_t ldh,
                          double bin, const double *q, uint32_t nq, double *d_G);
// The exact transform in steps: the plan (the q mesh on the device, sinc-digit planes for a mesh used
// again, count digits chosen from max_count; may synchronise), the launches (memsets and kernels only:
// can be captured in a CUDA graph), and the check of its flags.  d_G: ncols x nq FP64.
struct ExactLaunch {
  const unsigned long long *hist = nullptr;
  uint32_t ncols = 0, nh = 0, nq = 0, MT = 0, NT = 0, KT = 0;
  size_t ldh = 0, b_plane = 0;
  int digits = 0;  // count digits: 2, 3 or 4 (counts below 2^16, 2^24, 2^32)
  uint32_t ntile = 0;  // columns per N tile: 16 or 32
  const double *qv = nullptr;  // the q mesh on the device (sinc digits made on chip) ...
  double bin = 0;
  const uint8_t *A = nullptr;  // ... or the sinc-digit planes in HBM (a mesh used again)
  size_t a_plane = 0;
  uint8_t *B = nullptr;
  double *G = nullptr;
  int *flags = nullptr;
};
// planes: build the sinc-digit planes in HBM now (a plan whose launches are replayed) instead of on
// the mesh's second use.
int xns_tc_exact_plan(xns_ctx *ctx, const unsigned long long *d_hist, uint32_t ncols, uint32_t nh, size_t ldh, double bin,
                      const double *q, uint32_t nq, unsigned long long max_count, double *d_G, ExactLaunch *X,
                      bool planes = false);
int xns_tc_exact_enqueue(xns_ctx *ctx, const ExactLaunch &X);
int xns_tc_exact_check(xns_ctx *ctx, const ExactLaunch &X);
// Largest count of ncols histogram columns (synchronises).
int xns_tc_max_count(xns_ctx *ctx, const unsigned long long *d_hist, uint32_t ncols, uint32_t nh, size_t ldh,
                     unsigned long long *max_count);
// The whole contraction with integer digits and exact accumulation (tc_exact.cu).
// Angle-split FP64 sums G = sum_k (n(k) / r_k) sin(q r_k) and T = sum_k (n(k) / r_k^2) sin(q r_k), columns
// x nq each (hist_split.cu).
int xns_hist_transform_split(xns_ctx *ctx, const unsigned long long *d_hist, uint32_t ncols, uint32_t nh, size_t ldh,
                             double bin, const double *q, uint32_t nq, double *d_G, double *d_T);
int xns_tc_hist_transform_exact(xns_ctx *ctx, const unsigned long long *d_hist, uint32_t ncols, uint32_t nh, size_t ldh,
                             double bin, const double *q, uint32_t nq, double *d_G);
