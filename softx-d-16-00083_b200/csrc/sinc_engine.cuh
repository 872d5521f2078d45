// Sum of weighted sinc terms on a q mesh, shared by the exact Debye double sum (weights 1 per atom
// pair) and the allocation-free histogram transform (weight n_k per distance bin):
//
//   S_c(q_k) = sum_{records in class c} w sin(q_k r) / (q_k r + 1e-8)
//
// with the reference's +1e-8 (CalcFunctions.cpp:581, :861) kept: see "The +1e-8" below.
//
// Records (r, w) arrive in tiles of up to SE_TILE produced cooperatively by a Source in shared
// memory.  A lane owns a chunk of M consecutive q values, a slot of lanes walks the tile's records.
// On a uniform mesh q_k = q0 + k dq the lane seeds s_0 = sin(q_{k0} r) w/r and the difference
// d_0 = s_0 - s_{-1} = (sin(x) (1 - cos t) + cos(x) sin t) w/r (x = q_{k0} r, t = dq r) from an
// accurate sine and cosine of the FP64-reduced phase (xmath.cuh: the MUFU approximations would add
// coherently over the distance shells of a crystal), and runs the sine recurrence in Reinsch's
// difference form,
//   d_{k+1} = d_k - lam s_k,  s_{k+1} = s_k + d_{k+1},  lam = 4 sin^2(t/2),
// which is the Chebyshev recurrence s_{k+1} = 2cos(t) s_k - s_{k-1} with 2cos(t) kept as 2 - lam: lam
// carries full relative precision even for small t, so the phase does not drift the way a rounded
// 2cos(t) (error 2^-24 / sin t per step) would on fine q meshes.  A lane runs eight records side by
// side, as four packed pairs (f32x2.cuh): per (record, q) term one FFMA and one FADD for the sine, plus
// 7/8 FADD for the tree sum of the eight, no transcendental, in 13 instructions per eight terms.  The
// next eight records' seeds are computed in the same straight-line block as this recurrence, so that
// their latency overlaps its steps.
//
// Accumulation: FP32 sums over at most SE_FP32_GROUPS groups of eight records, then per-thread FP64
// totals in shared memory, then FP64 per-CTA partial sums reduced in the epilogue.  1/q_k is applied
// in the epilogue.  A mesh that is not uniform takes an accurate sine per term (DIRECT).
//
// The +1e-8.  sin(q r)/(q r + 1e-8) = sin(q r)/(q r) - 1e-8 sin(q r)/(q r)^2 + O(1e-16): the second
// term is a relative 1e-8/(q r) of each term, below FP32 resolution, but at the deepest minima of a
// pattern (I down to 1e-5 of its maximum) it adds coherently to ~3e-5 of I.  The engine therefore
// adds every record's w / r^2 into a coarse distance histogram (bin >= 0.05 A) as it builds the
// record, sinc_eps_kernel forms T_c(q) = sum_b H_c[b] sin(q r_b) from it in FP64, and the epilogue
// subtracts 1e-8 T_c(q) / q^2.  At the q where the term matters (q r_b <~ 5) the coarse bins change
// T by a relative (q bin)^2 / 24 < 1e-4.
#pragma once
#include <math.h>

#include <algorithm>

#include "f32x2.cuh"
#include "xmath.cuh"
#include "xns_internal.cuh"

namespace xns_sinc {

constexpr int SE_THREADS = 128;
// CTAs per SM the register allocation is sized for (168 registers a thread).
constexpr int SE_MIN_CTAS = 3;
// Records per tile.  With 16 lanes per slot (1024 q) a lane takes 6 groups of eight records per tile;
// the FP64 totals take 64 KB, the records 9 KB: three CTAs (12 warps) share an SM.
constexpr int SE_TILE = 384;
// q values per lane: M_UNIFORM for the recurrence (a seed costs ~30 instructions, the recurrence
// 1.6 issue slots per term), M_DIRECT for the per-term sine of a non-uniform mesh.
constexpr int SE_M_UNIFORM = 64;
constexpr int SE_M_DIRECT = 16;
// Records a lane runs side by side (four packed pairs).
constexpr int SE_GROUP = 8;
// Record groups a lane sums in FP32 before the sums go to FP64 (48 records; the error of these FP32
// sums is the largest term of the error budget at the deepest minima of a pattern).
constexpr int SE_FP32_GROUPS = 6;
// The +1e-8 histogram: bins of at least EPS_BIN_MIN, at most EPS_NB_MAX of them.
constexpr double EPS_BIN_MIN = 0.05;
constexpr uint32_t EPS_NB_MAX = 16384;
constexpr double SINC_EPS = 1e-8;  // CalcFunctions.cpp:581, :861

struct PairRec {
  double r;    // distance (FP64)
  float w;     // weight / r; 0 for a record that does not count
  float a;     // w sin(t),            t = dq r
  float b;     // w (1 - cos t) = 2 w sin^2(t/2)
  float lam;   // 4 sin^2(t/2) = 2 - 2 cos(t)
};

__device__ __forceinline__ PairRec null_rec() { return PairRec{1.0, 0.f, 0.f, 0.f, 0.f}; }

struct SincParams {
  double q0, dq;      // uniform mesh
  const double *q;    // the mesh itself (DIRECT)
  uint32_t nq;
  uint32_t ncls;
  unsigned long long ntiles;
  double *partial;    // [gridDim.x][ncls][nq] FP64, zeroed
  uint32_t shard = 0, nshard = 1;  // this launch sums the tiles w with w % nshard == shard
  // the +1e-8 histogram [ncls][eps_nb] (null: not kept), bin width 1 / eps_inv_bw
  double *eps_hist = nullptr;
  uint32_t eps_nb = 0;
  double eps_inv_bw = 0;
};

// The record of distance r > 0 and weight w of class cls; adds w / r^2 to the +1e-8 histogram.
__device__ __forceinline__ PairRec make_rec(const SincParams &p, uint32_t cls, double r, double w) {
  PairRec rec;
  double sh, ch;
  xns_math::xns_sincos64(0.5 * p.dq * r, &sh, &ch);
  const double wr = w / r;
  rec.r = r;
  rec.w = (float)wr;
  rec.a = (float)(2.0 * sh * ch * wr);
  rec.b = (float)(2.0 * sh * sh * wr);
  rec.lam = (float)(4.0 * sh * sh);
  if (p.eps_hist) {
    const uint32_t k = (uint32_t)fmin(r * p.eps_inv_bw, (double)(p.eps_nb - 1));
    atomicAdd(p.eps_hist + (size_t)cls * p.eps_nb + k, wr / r);
  }
  return rec;
}

// Shared memory: [M][SE_THREADS] FP64 totals (one column per thread), then SE_TILE records, then the
// Source's own staging area.
template <int M, bool DIRECT, class Src>
__global__ void __launch_bounds__(SE_THREADS, SE_MIN_CTAS) sinc_tiles_kernel(SincParams p, Src src, int lanes_per_slot) {
  extern __shared__ double acc64[];
  constexpr int ncol = SE_THREADS;
  PairRec *pr = reinterpret_cast<PairRec *>(acc64 + M * ncol);
  void *stage = reinterpret_cast<void *>(pr + SE_TILE);

  const int tid = threadIdx.x, col = tid;
  const int nslots = SE_THREADS / lanes_per_slot;
  const int slot = tid / lanes_per_slot;
  const uint32_t k0 = (uint32_t)(tid % lanes_per_slot) * M;
  const bool active = k0 < p.nq;
  const double qk0 = p.q0 + (double)k0 * p.dq;
#pragma unroll
  for (int k = 0; k < M; k++) acc64[k * ncol + col] = 0.0;
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
          if (k0 + k < p.nq) atomicAdd(dst + k, acc64[k * ncol + col]);
          acc64[k * ncol + col] = 0.0;
        }
      }
      cur = c;
    }
    const int n = src.fill(w, pr, stage, p, (uint32_t)c);  // ends with __syncthreads()
    float blk[M];
#pragma unroll
    for (int k = 0; k < M; k++) blk[k] = 0.f;
    if (active && DIRECT) {
      int nblk = 0;  // record groups in blk
      // a lane takes four records per step: e, e + S, e + 2S, e + 3S (S = slots)
      for (int e = slot; e < n; e += 4 * nslots) {
        PairRec R[4];
#pragma unroll
        for (int g = 0; g < 4; g++) R[g] = e + g * nslots < n ? pr[e + g * nslots] : null_rec();
        if (R[0].w == 0.f && R[1].w == 0.f && R[2].w == 0.f && R[3].w == 0.f) continue;
        if (nblk == SE_FP32_GROUPS) {  // FP32 sums stay short
#pragma unroll
          for (int k = 0; k < M; k++) {
            acc64[k * ncol + col] += (double)blk[k];
            blk[k] = 0.f;
          }
          nblk = 0;
        }
        nblk++;
        float wr[4];
#pragma unroll
        for (int g = 0; g < 4; g++) wr[g] = R[g].w;
#pragma unroll
        for (int k = 0; k < M; k++) {
          float t = 0.f;
#pragma unroll
          for (int g = 0; g < 4; g++) t += xns_math::xns_sin(qd[k] * R[g].r) * wr[g];
          blk[k] += t;
        }
      }
    } else if (active) {
      // a lane takes SE_GROUP records per step: e, e + S, ..., e + (SE_GROUP - 1) S (S = slots); the
      // next group's seeds are computed in one straight-line block with this group's recurrence
      constexpr int G = SE_GROUP, H = SE_GROUP / 2;
      float s[G], d[G], lam[G];
      auto seeds = [&](int e0, float *so, float *dO, float *lo_) {
#pragma unroll
        for (int g = 0; g < G; g++) {
          const PairRec R = e0 + g * nslots < n ? pr[e0 + g * nslots] : null_rec();
          float sn, cs;
          xns_math::xns_sincos(qk0 * R.r, &sn, &cs);
          so[g] = sn * R.w;
          dO[g] = fmaf(cs, R.a, sn * R.b);
          lo_[g] = R.lam;
        }
      };
      seeds(slot, s, d, lam);
      int nblk = 0;  // record groups in blk
      for (int e = slot; e < n; e += G * nslots) {
        if (nblk == SE_FP32_GROUPS) {  // FP32 sums stay short
#pragma unroll
          for (int k = 0; k < M; k++) {
            acc64[k * ncol + col] += (double)blk[k];
            blk[k] = 0.f;
          }
          nblk = 0;
        }
        nblk++;
        using namespace xns_f2;
        f2 S[H], D[H], L[H];
#pragma unroll
        for (int h = 0; h < H; h++) {  // packed pairs of records (h, h + H)
          S[h] = pack(s[h], s[h + H]);
          D[h] = pack(d[h], d[h + H]);
          L[h] = pack(-lam[h], -lam[h + H]);
        }
        seeds(e + G * nslots, s, d, lam);
        {
          const f2 u = add(add(S[0], S[1]), add(S[2], S[3]));
          blk[0] += lo(u) + hi(u);
        }
        // the recurrence on packed pairs: the same roundings as scalar FFMA / FADD, half the instructions
#pragma unroll
        for (int k = 1; k < M; k++) {
#pragma unroll
          for (int h = 0; h < H; h++) D[h] = xns_f2::fma(L[h], S[h], D[h]);
#pragma unroll
          for (int h = 0; h < H; h++) S[h] = add(S[h], D[h]);
          const f2 u = add(add(S[0], S[1]), add(S[2], S[3]));
          blk[k] += lo(u) + hi(u);
        }
      }
    }
    if (active) {
#pragma unroll
      for (int k = 0; k < M; k++) acc64[k * ncol + col] += (double)blk[k];
    }
    __syncthreads();
  }
  if (cur >= 0 && active) {
    double *dst = p.partial + ((size_t)blockIdx.x * p.ncls + cur) * p.nq + k0;
#pragma unroll
    for (int k = 0; k < M; k++)
      if (k0 + k < p.nq) atomicAdd(dst + k, acc64[k * ncol + col]);
  }
}

// T[c][iq] = sum_b H[c][b] sin(q_iq r_b), r_b = (b + 0.5) bin: the +1e-8 sum (H holds w / r^2).  A
// thread owns one q and EPS_RUN bins, stepping the phase by an FP64 rotation.
constexpr uint32_t EPS_RUN = 256;
__global__ void sinc_eps_kernel(const double *__restrict__ H, uint32_t nb, double bin, double q0, double dq,
                                const double *__restrict__ qmesh, uint32_t nq, double *__restrict__ T);

// Reduction of the per-CTA FP64 partial sums plus the calc-function epilogue: 1/q, weights, self
// term, 1/Ntot, polarisation factor and the sum over parts (CalcFunctions.cpp:592-625 and 733-755 for
// the Debye sums, :872-906 for the histogram transform).  Classes are part * P + t.
// out: [total | parts] when nparts > 1, else [total].  over_q: the partial sums still need the 1/q
// (and, with eps_t, the +1e-8 term -1e-8 eps_t[c][iq] / q^2).
__global__ void sinc_epilogue_kernel(const double *__restrict__ partial, int grid, uint32_t ncls, uint32_t nel,
                                     uint32_t nparts, uint32_t nblocks, const uint32_t *__restrict__ pair_a,
                                     const uint32_t *__restrict__ pair_b, const double *__restrict__ w,
                                     const uint32_t *__restrict__ n_el_block, double q0, double dq,
                                     const double *__restrict__ qmesh, uint32_t nq, uint32_t ntot, int polar, double lambda,
                                     int over_q, int self_term, const double *__restrict__ eps_t, double *__restrict__ out);

// Bin count and width of the +1e-8 histogram for distances up to rmax.
inline void eps_layout(double rmax, uint32_t nb_max, uint32_t *nb, double *bin) {
  double b = std::max(EPS_BIN_MIN, rmax / (double)(nb_max - 1));
  *bin = b;
  *nb = std::min(nb_max, (uint32_t)(rmax / b) + 2);
}

size_t sinc_smem_bytes(int M, int lanes_per_slot, size_t stage_bytes);

// Launches sinc_tiles_kernel with the persistent grid and zeroed partial sums (and, with rmax > 0,
// a zeroed +1e-8 histogram for distances up to rmax, then sinc_eps_kernel into SLOT_EPS_T); returns
// the status and the grid size used.
template <int M, bool DIRECT, class Src>
int launch_sinc(xns_ctx *ctx, const SincParams &p, const Src &src, int lanes, size_t stage_bytes, double rmax,
                int *grid_out) {
  const size_t smem = sinc_smem_bytes(M, lanes, stage_bytes);
  auto kern = sinc_tiles_kernel<M, DIRECT, Src>;
  XNS_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sinc_smem_bytes(M, SE_THREADS, stage_bytes)));
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
  double ebin = 0;
  if (rmax > 0) {
    eps_layout(rmax, EPS_NB_MAX, &pp.eps_nb, &ebin);
    pp.eps_inv_bw = 1.0 / ebin;
    const size_t hb = sizeof(double) * p.ncls * pp.eps_nb;
    if ((st = xns_scratch(ctx, SLOT_EPS_HIST, hb, &d))) return st;
    XNS_CUDA(ctx, cudaMemsetAsync(d, 0, hb, ctx->stream));
    pp.eps_hist = (double *)d;
  }
  if (p.ntiles) {
    kern<<<(unsigned)grid, SE_THREADS, smem, ctx->stream>>>(pp, src, lanes);
    XNS_LAUNCHED(ctx);
  }
  if (rmax > 0) {
    const size_t tb = sizeof(double) * p.ncls * p.nq;
    if ((st = xns_scratch(ctx, SLOT_EPS_T, tb, &d))) return st;
    XNS_CUDA(ctx, cudaMemsetAsync(d, 0, tb, ctx->stream));
    dim3 g((p.nq + 127) / 128, (pp.eps_nb + EPS_RUN - 1) / EPS_RUN, p.ncls);
    sinc_eps_kernel<<<g, 128, 0, ctx->stream>>>(pp.eps_hist, pp.eps_nb, ebin, p.q0, p.dq, DIRECT ? p.q : nullptr, p.nq,
                                                (double *)d);
    XNS_LAUNCHED(ctx);
  }
  *grid_out = (int)grid;
  return XNS_OK;
}

// Chooses M and the lanes per slot for nq and launches; DIRECT when the mesh is not uniform.
// rmax: the largest distance of a record (> 0 keeps the +1e-8 term, see the top of this file).
template <class Src>
int run_sinc(xns_ctx *ctx, SincParams p, const Src &src, size_t stage_bytes, bool uniform, double rmax, int *grid_out) {
  const int M = uniform ? SE_M_UNIFORM : SE_M_DIRECT;
  const uint32_t chunks = (p.nq + M - 1) / M;
  int lanes = 1;
  while (lanes < (int)chunks) lanes <<= 1;
  if (lanes > SE_THREADS) return xns_fail(ctx, XNS_ERR_ARG, "too many q points for one call");
  if (uniform) return launch_sinc<SE_M_UNIFORM, false>(ctx, p, src, lanes, stage_bytes, rmax, grid_out);
  return launch_sinc<SE_M_DIRECT, true>(ctx, p, src, lanes, stage_bytes, rmax, grid_out);
}

// Uploads pair_a, pair_b, n_el_block and the q mesh for the epilogue and runs it.  partial: grid x ncls
// x nq sums (null: the engine's per-CTA partials); over_q: the sums are sum w sin(q r)/r and still
// need the 1/q (the engine's), otherwise they are already sum w sin(q r)/(q r + 1e-8).  eps_t: the
// engine's +1e-8 sums (SLOT_EPS_T) or null.
int sinc_epilogue(xns_ctx *ctx, int grid, uint32_t ncls, uint32_t nel, uint32_t nblocks, const uint32_t *n_el_block,
                  const double *q, uint32_t nq, bool uniform, double q0, double dq, const double *d_w, uint32_t ntot,
                  int polar, double lambda, double *d_out, const double *partial = nullptr, bool over_q = true,
                  bool self_term = true, const double *eps_t = nullptr);
// The q mesh as a device array (valid until the next call on the context).
int sinc_upload_q(xns_ctx *ctx, const double *q, uint32_t nq, const double **d_q);

}  // namespace xns_sinc
