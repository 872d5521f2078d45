// Sum of weighted sinc terms on a q mesh, shared by the exact Debye double sum (weights 1 per atom
// pair) and the histogram transform (weight n_k per distance bin):
//
//   S_c(q_k) = sum_{records in class c} w * sin(q_k r) / (q_k r)
//
// Records (r, w) arrive in tiles of up to SE_TILE produced cooperatively by a Source in shared
// memory.  A lane owns a chunk of M consecutive q values, a slot of lanes walks the tile's records.
// On a uniform mesh q_k = q0 + k dq the lane seeds s_0 = sin(q_{k0} r) w/r and the difference
// d_0 = s_0 - s_{-1} = 2 sin(t/2) cos(q_{k0} r - t/2) w/r (t = dq r) from an accurate sine and cosine
// of the FP64 phase (xmath.cuh; the MUFU approximations would add coherently over the distance shells
// of a crystal) and runs the sine recurrence in Reinsch's difference form,
//   d_{k+1} = d_k - lam s_k,  s_{k+1} = s_k + d_{k+1},  lam = 4 sin^2(t/2),
// which is the Chebyshev recurrence s_{k+1} = 2cos(t) s_k - s_{k-1} with 2cos(t) kept as 2 - lam: lam
// carries full relative precision even for small t, so the phase does not drift the way a rounded
// 2cos(t) (error 2^-24 / sin t per step) would on fine q meshes.  A lane runs four records side by
// side, as two packed pairs (f32x2.cuh): per (record, q) term one FFMA and one FADD for the sine, plus
// 3/4 FADD for the pairwise sum of the four, no transcendental, in 7 instructions per four terms.  Sums run in FP32 over SE_FP32_GROUPS groups and are then added to
// per-thread FP64 totals in shared memory (compensated block accumulation); CTAs then reduce in FP64
// in the epilogue.  1/q_k is applied in the epilogue.  A mesh that is not uniform takes an accurate
// sine per term (DIRECT).
#pragma once
#include <math.h>

#include <algorithm>

#include "f32x2.cuh"
#include "xmath.cuh"
#include "xns_internal.cuh"

namespace xns_sinc {

constexpr int SE_THREADS = 128;
// Records per tile.  With M = 64 the FP64 totals take 64 KB of shared memory per CTA; 384 records
// (9 KB) keep a CTA under a third of the SM's shared memory, so that three CTAs (12 warps, at most 168
// registers a thread) share an SM.
constexpr int SE_TILE = 384;
// q values per lane: M_UNIFORM for the recurrence (a seed costs ~30 instructions, the recurrence 2.75
// per term), M_DIRECT for the per-term sine of a non-uniform mesh.
constexpr int SE_M_UNIFORM = 64;
constexpr int SE_M_DIRECT = 16;
// Record groups (4 records each) a lane sums in FP32 before adding the sums to its FP64 totals.  A
// lane adds each group's terms to a running FP32 sum, so the rounding error grows with the length of
// that sum; with the large cancellation at the minima of I(q) (sum of |terms| ~10^3 x the result) 16
// records keep the FP32 summation error within ~3x of the FP32 rounding of the terms themselves.
constexpr int SE_FP32_GROUPS = 4;

struct PairRec {
  double r;      // distance (FP64)
  float w_r;     // weight / r; 0 for a record that does not count
  float lam;     // 4 sin^2(dq r / 2) = 2 - 2 cos(dq r)
  float h2;      // 2 sin(dq r / 2)
  float ch;      // cos(dq r / 2)
};

__device__ __forceinline__ PairRec make_rec(double r, double w, double dq) {
  PairRec rec;
  rec.r = r;
  rec.w_r = (float)(w / r);
  float s, c;
  xns_math::xns_sincos(0.5 * dq * r, &s, &c);
  rec.lam = 4.f * s * s;
  rec.h2 = 2.f * s;
  rec.ch = c;
  return rec;
}

__device__ __forceinline__ PairRec null_rec() { return PairRec{1.0, 0.f, 0.f, 0.f, 1.f}; }

struct SincParams {
  double q0, dq;      // uniform mesh
  const double *q;    // the mesh itself (DIRECT)
  uint32_t nq;
  uint32_t ncls;
  unsigned long long ntiles;
  double *partial;    // [gridDim.x][ncls][nq] FP64, zeroed
  uint32_t shard = 0, nshard = 1;  // this launch sums the tiles w with w % nshard == shard
};

// Shared memory: [M][SE_THREADS] FP64 totals (one column per thread), then SE_TILE records, then the
// Source's own staging area.
template <int M, bool DIRECT, class Src>
__global__ void __launch_bounds__(SE_THREADS, 3) sinc_tiles_kernel(SincParams p, Src src, int lanes_per_slot) {
  extern __shared__ double acc64[];
  PairRec *pr = reinterpret_cast<PairRec *>(acc64 + M * SE_THREADS);
  void *stage = reinterpret_cast<void *>(pr + SE_TILE);

  const int tid = threadIdx.x;
  const int nslots = SE_THREADS / lanes_per_slot;
  const int slot = tid / lanes_per_slot;
  const uint32_t k0 = (uint32_t)(tid % lanes_per_slot) * M;
  const bool active = k0 < p.nq;
  const double qk0 = p.q0 + (double)k0 * p.dq;
#pragma unroll
  for (int k = 0; k < M; k++) acc64[k * SE_THREADS + tid] = 0.0;
  double qd[DIRECT ? M : 1];
  if (DIRECT) {
#pragma unroll
    for (int k = 0; k < (DIRECT ? M : 1); k++) qd[k] = (k0 + k < p.nq) ? p.q[k0 + k] : 0.0;
  }

  int cur = -1;
  for (unsigned long long w = p.shard + (unsigned long long)p.nshard * blockIdx.x; w < p.ntiles;
       w += (unsigned long long)p.nshard * gridDim.x) {
    const int c = (int)src.cls(w);
    if (c != cur) {  // flush the previous class's FP64 totals to this CTA's slice
      if (cur >= 0 && active) {
        double *dst = p.partial + ((size_t)blockIdx.x * p.ncls + cur) * p.nq + k0;
#pragma unroll
        for (int k = 0; k < M; k++) {
          if (k0 + k < p.nq) atomicAdd(dst + k, acc64[k * SE_THREADS + tid]);
          acc64[k * SE_THREADS + tid] = 0.0;
        }
      }
      cur = c;
    }
    const int n = src.fill(w, pr, stage, p.dq);  // ends with __syncthreads()
    if (active) {
      float blk[M];
#pragma unroll
      for (int k = 0; k < M; k++) blk[k] = 0.f;
      int nblk = 0;  // record groups in blk
      // a lane takes four records per step: e, e + S, e + 2S, e + 3S (S = slots)
      for (int e = slot; e < n; e += 4 * nslots) {
        PairRec R[4];
#pragma unroll
        for (int g = 0; g < 4; g++) R[g] = e + g * nslots < n ? pr[e + g * nslots] : null_rec();
        if (R[0].w_r == 0.f && R[1].w_r == 0.f && R[2].w_r == 0.f && R[3].w_r == 0.f) continue;
        if (nblk == SE_FP32_GROUPS) {  // FP32 sums stay short: move them to the FP64 totals
#pragma unroll
          for (int k = 0; k < M; k++) {
            acc64[k * SE_THREADS + tid] += (double)blk[k];
            blk[k] = 0.f;
          }
          nblk = 0;
        }
        nblk++;
        if (DIRECT) {
#pragma unroll
          for (int k = 0; k < M; k++) {
            float t = 0.f;
#pragma unroll
            for (int g = 0; g < 4; g++) t += xns_math::xns_sin(qd[k] * R[g].r) * R[g].w_r;
            blk[k] += t;
          }
        } else {
          // seeds: s_0 = sin(x), d_0 = s_0 - s_{-1} = 2 sin(t/2) cos(x - t/2) with x = q_{k0} r, t = dq r
          float s[4], d[4], lam[4];
#pragma unroll
          for (int g = 0; g < 4; g++) {
            float sx, cx;
            xns_math::xns_sincos(qk0 * R[g].r, &sx, &cx);
            s[g] = sx * R[g].w_r;
            d[g] = R[g].h2 * fmaf(cx, R[g].ch, sx * (0.5f * R[g].h2)) * R[g].w_r;
            lam[g] = R[g].lam;
          }
          // the recurrence on packed pairs of records (0, 1) and (2, 3): the same roundings as scalar
          // FFMA / FADD, half the instructions
          using namespace xns_f2;
          f2 S01 = pack(s[0], s[1]), S23 = pack(s[2], s[3]), D01 = pack(d[0], d[1]), D23 = pack(d[2], d[3]);
          const f2 L01 = pack(-lam[0], -lam[1]), L23 = pack(-lam[2], -lam[3]);
          blk[0] += (s[0] + s[2]) + (s[1] + s[3]);
#pragma unroll
          for (int k = 1; k < M; k++) {
            D01 = xns_f2::fma(L01, S01, D01);
            D23 = xns_f2::fma(L23, S23, D23);
            S01 = add(S01, D01);
            S23 = add(S23, D23);
            const f2 u = add(S01, S23);  // (s0 + s2, s1 + s3)
            blk[k] += lo(u) + hi(u);
          }
        }
      }
#pragma unroll
      for (int k = 0; k < M; k++) acc64[k * SE_THREADS + tid] += (double)blk[k];
    }
    __syncthreads();
  }
  if (cur >= 0 && active) {
    double *dst = p.partial + ((size_t)blockIdx.x * p.ncls + cur) * p.nq + k0;
#pragma unroll
    for (int k = 0; k < M; k++)
      if (k0 + k < p.nq) atomicAdd(dst + k, acc64[k * SE_THREADS + tid]);
  }
}

// Reduction of the per-CTA FP64 partial sums plus the calc-function epilogue: 1/q, weights, self
// term, 1/Ntot, polarisation factor and the sum over parts (CalcFunctions.cpp:592-625 and 733-755 for
// the Debye sums, :872-906 for the histogram transform).  Classes are part * P + t.
// out: [total | parts] when nparts > 1, else [total].  over_q: the partial sums still need the 1/q.
__global__ void sinc_epilogue_kernel(const double *__restrict__ partial, int grid, uint32_t ncls, uint32_t nel,
                                     uint32_t nparts, uint32_t nblocks, const uint32_t *__restrict__ pair_a,
                                     const uint32_t *__restrict__ pair_b, const double *__restrict__ w,
                                     const uint32_t *__restrict__ n_el_block, double q0, double dq,
                                     const double *__restrict__ qmesh, uint32_t nq, uint32_t ntot, int polar, double lambda,
                                     int over_q, int self_term, double *__restrict__ out);

// Launches sinc_tiles_kernel with the persistent grid and zeroed partial sums; returns the status
// and the grid size used.
template <int M, bool DIRECT, class Src>
int launch_sinc(xns_ctx *ctx, const SincParams &p, const Src &src, int lanes, size_t stage_bytes, int *grid_out) {
  const size_t smem = sizeof(double) * M * SE_THREADS + sizeof(PairRec) * SE_TILE + stage_bytes;
  auto kern = sinc_tiles_kernel<M, DIRECT, Src>;
  XNS_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  XNS_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, SE_THREADS, smem));
  const unsigned long long mine = p.nshard > 1 ? (p.ntiles + p.nshard - 1) / p.nshard : p.ntiles;
  unsigned long long grid = std::min<unsigned long long>(mine, (unsigned long long)ctx->num_sms * std::max(per_sm, 1));
  if (grid == 0) grid = 1;
  SincParams pp = p;
  void *d;
  int st;
  size_t bytes = sizeof(double) * grid * p.ncls * p.nq;
  if ((st = xns_scratch(ctx, SLOT_PARTIAL, bytes, &d))) return st;
  XNS_CUDA(ctx, cudaMemsetAsync(d, 0, bytes, ctx->stream));
  pp.partial = (double *)d;
  if (p.ntiles) {
    kern<<<(unsigned)grid, SE_THREADS, smem, ctx->stream>>>(pp, src, lanes);
    XNS_LAUNCHED(ctx);
  }
  *grid_out = (int)grid;
  return XNS_OK;
}

// Chooses M and the lanes per slot for nq and launches; DIRECT when the mesh is not uniform.
template <class Src>
int run_sinc(xns_ctx *ctx, SincParams p, const Src &src, size_t stage_bytes, bool uniform, int *grid_out) {
  const int M = uniform ? SE_M_UNIFORM : SE_M_DIRECT;
  const uint32_t chunks = (p.nq + M - 1) / M;
  int lanes = 1;
  while (lanes < (int)chunks) lanes <<= 1;
  if (lanes > SE_THREADS) return xns_fail(ctx, XNS_ERR_ARG, "too many q points for one call");
  if (uniform) return launch_sinc<SE_M_UNIFORM, false>(ctx, p, src, lanes, stage_bytes, grid_out);
  return launch_sinc<SE_M_DIRECT, true>(ctx, p, src, lanes, stage_bytes, grid_out);
}

// Uploads pair_a, pair_b, n_el_block and the q mesh for the epilogue and runs it.  partial: grid x ncls
// x nq sums (null: the engine's per-CTA partials); over_q: the sums are sum w sin(q r)/r and still
// need the 1/q (the engine's), otherwise they are already sum w sin(q r)/(q r + 1e-8).
int sinc_epilogue(xns_ctx *ctx, int grid, uint32_t ncls, uint32_t nel, uint32_t nblocks, const uint32_t *n_el_block,
                  const double *q, uint32_t nq, bool uniform, double q0, double dq, const double *d_w, uint32_t ntot,
                  int polar, double lambda, double *d_out, const double *partial = nullptr, bool over_q = true,
                  bool self_term = true);
// The q mesh as a device array (valid until the next call on the context).
int sinc_upload_q(xns_ctx *ctx, const double *q, uint32_t nq, const double **d_q);

}  // namespace xns_sinc
