// Histogram -> I(q) sums by angle splitting (the contraction of calcInt1DHist, CalcFunctions.cpp:
// 846-868, and calcIntHistKernel*, CalcFunctionsCUDA.cu:923-1045), in FP64 with no sinc matrix.
//
// The reference sums n(k) sin(q r_k) / (q r_k + 1e-8) over the bins, r_k = (k + 0.5) bin.  To first
// order in the 1e-8 (the next term is below 1e-14 of the sum's terms for every populated bin),
//   sum_k n(k) sin(q r_k) / (q r_k + eps) = G(q) / q - eps T(q) / q^2,
//   G(q) = sum_k (n(k) / r_k) sin(q r_k),   T(q) = sum_k (n(k) / r_k^2) sin(q r_k),
// which is what the shared epilogue (sinc_engine.cu, over_q with eps_t) expects.  Writing the bin
// k = 64 h + l as r_k = R_h + r_l with R_h = 64 h bin and r_l = (l + 0.5) bin,
//   sin(q r_k) = sin(q R_h) cos(q r_l) + cos(q R_h) sin(q r_l),
// so with g_h,l = n(64 h + l) / r_k,
//   G(q) = sum_h [ sin(q R_h) sum_l g_h,l cos(q r_l) + cos(q R_h) sum_l g_h,l sin(q r_l) ].
// The inner sums are a product with K = 64 against two tables of 64 cosines and sines per q; the
// outer weights sin / cos(q R_h) follow h by a rotation.  Per (q, bin, column): two FP64 FMAs for G
// and two FP32 FMAs for T (the 1e-8 term needs ~1e-3 relative; FP32 sums on the FP32 pipe, beside
// the FP64 pipe), instead of a sinc value and its digits per element.
//
// split_sum_kernel: a CTA takes 64 q (the tables, 96 KB, in shared memory) and a range of blocks h;
// each thread takes 4 q x CB columns and every 16th block of the range.  Partial sums per CTA are
// reduced over the CTA's threads in a fixed order and over the h ranges by split_reduce_kernel, so
// the result does not depend on scheduling.
#include <string.h>

#include <algorithm>
#include <vector>

#include "f32x2.cuh"
#include "tc_gemm.cuh"
#include "xmath.cuh"
#include "xns_internal.cuh"

namespace {

constexpr int SQ = 64;    // q per CTA
constexpr int SLO = 64;   // bins per block h (the K of the inner product)
constexpr int ST = 256;   // threads per CTA
constexpr int SHL = 16;   // block lanes per CTA (threads with the same 4 q take every 16th block)
constexpr int TQ = 4;     // q per thread
constexpr int CBMAX = 4;  // columns per pass
static_assert(SQ == TQ * (ST / SHL), "a CTA's threads cover its q tile");

// Column stride of the G tables: 1, 2 or 4 (three columns are padded to four for 16-byte loads).
__host__ __device__ constexpr int gstride(int cb) { return cb == 3 ? 4 : cb; }

// Tables per q tile qt: A64[qt][0][l][j] = cos(q r_l), A64[qt][1][l][j] = sin(q r_l) for q the tile's
// j-th value (0 past nq), A32 the same rounded to float; qv the padded mesh.
__global__ void split_tables_kernel(const double *__restrict__ qmesh, uint32_t nq, uint32_t nq_pad,
                                    double bin, double *__restrict__ A64, float *__restrict__ A32,
                                    double *__restrict__ qv) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;  // (q, l) with l fastest
  if (i >= nq_pad * SLO) return;
  const uint32_t iq = i / SLO, l = i % SLO;
  const double q = iq < nq ? qmesh[iq] : 0.0;
  if (l == 0) qv[iq] = q;
  double s, c;
  xns_math::xns_sincos64_acc(q * ((l + 0.5) * bin), &s, &c);
  const size_t o = (size_t)(iq / SQ) * 2 * SLO * SQ + (size_t)l * SQ + iq % SQ;
  A64[o] = c;
  A64[o + SLO * SQ] = s;
  A32[o] = (float)c;
  A32[o + SLO * SQ] = (float)s;
}

// G1[k][c] = n_c(k) / r_k and G2[k][c] = n_c(k) / r_k^2 (float) for the columns c0 .. c0 + cb - 1 of
// this pass, zero past nh and in the padding.
__global__ void split_weights_kernel(const unsigned long long *__restrict__ hist, size_t ldh, uint32_t c0, uint32_t cb,
                                     uint32_t gs, uint32_t nh, uint32_t nh_pad, double bin, double *__restrict__ G1,
                                     float *__restrict__ G2) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nh_pad) return;
  const double r = (k + 0.5) * bin;
  for (uint32_t c = 0; c < gs; c++) {
    const double n = (c < cb && k < nh) ? (double)hist[(size_t)(c0 + c) * ldh + k] : 0.0;
    const double g = n / r;
    G1[(size_t)k * gs + c] = g;
    G2[(size_t)k * gs + c] = (float)(g / r);
  }
}

struct SplitArgs {
  const double *A64;
  const float *A32;
  const double *G1;
  const float *G2;
  const double *qv;
  double *part;  // [split][2][CB][nq_pad]: G sums, then T sums
  uint32_t nhi, nq_pad, nsplit, hi_per_split;
  double blk;  // 64 bin
};

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Shared memory of split_sum_kernel: the q tile's tables (FP64 cos, sin; FP32 cos, sin: 96 KB), then two
// stages of one step's G rows (16 blocks x 64 bins x GS columns, FP64 and FP32).
__host__ __device__ constexpr size_t split_stage_bytes(int gs) { return (size_t)SHL * SLO * gs * (8 + 4); }
__host__ __device__ constexpr size_t split_smem_bytes(int gs) {
  return (size_t)2 * SLO * SQ * (8 + 4) + 2 * split_stage_bytes(gs);
}

// A thread's q: 2g, 2g + 1, 32 + 2g, 33 + 2g of the tile (g = thread % 16), so that the 16 threads of a
// half warp read 256 contiguous bytes per table load.
__device__ __forceinline__ uint32_t split_q(uint32_t g, int t) { return (t < 2 ? 0u : 32u) + 2 * g + (t & 1); }

template <int CB>
__global__ void __launch_bounds__(ST, 1) split_sum_kernel(SplitArgs a) {
  constexpr int GS = gstride(CB);
  constexpr uint32_t G1N = SHL * SLO * GS;  // doubles (and floats) of one step's G rows
  extern __shared__ __align__(16) unsigned char smem[];
  double *c64 = reinterpret_cast<double *>(smem);  // [SLO][SQ] cos, then [SLO][SQ] sin
  float *c32 = reinterpret_cast<float *>(c64 + 2 * SLO * SQ);
  double *gs64 = reinterpret_cast<double *>(c32 + 2 * SLO * SQ);  // [stage][G1N]
  float *gs32 = reinterpret_cast<float *>(gs64 + 2 * G1N);           // [stage][G1N]
  const uint32_t qt = blockIdx.x / a.nsplit, sp = blockIdx.x % a.nsplit;
  const uint32_t hb = sp * a.hi_per_split, he = min(hb + a.hi_per_split, a.nhi);
  const uint32_t nsteps = (he - hb + SHL - 1) / SHL;
  // one step's G rows: blocks hb + SHL s .. + SHL - 1 are contiguous in the tables; blocks past the
  // last one are not copied (their threads do not read them)
  auto prefetch = [&](uint32_t s, uint32_t stage) {
    const uint32_t h0 = hb + s * SHL, nrow = min((uint32_t)SHL, a.nhi - h0);
    const uint32_t n1 = nrow * SLO * GS / 2, n2 = nrow * SLO * GS / 4;  // 16-byte pieces
    const double *g1 = a.G1 + (size_t)h0 * SLO * GS;
    const float *g2 = a.G2 + (size_t)h0 * SLO * GS;
    double *d1 = gs64 + stage * G1N;
    float *d2 = gs32 + stage * G1N;
    for (uint32_t i = threadIdx.x; i < n1; i += ST) cp_async16(d1 + 2 * i, g1 + 2 * i);
    for (uint32_t i = threadIdx.x; i < n2; i += ST) cp_async16(d2 + 4 * i, g2 + 4 * i);
    cp_async_commit();
  };
  if (nsteps) prefetch(0, 0);
  {  // the tile's tables: 64 KB FP64, 32 KB FP32
    const double2 *src = reinterpret_cast<const double2 *>(a.A64 + (size_t)qt * 2 * SLO * SQ);
    double2 *dst = reinterpret_cast<double2 *>(c64);
    for (uint32_t i = threadIdx.x; i < 2 * SLO * SQ / 2; i += ST) dst[i] = src[i];
    const float4 *s32 = reinterpret_cast<const float4 *>(a.A32 + (size_t)qt * 2 * SLO * SQ);
    float4 *d32 = reinterpret_cast<float4 *>(c32);
    for (uint32_t i = threadIdx.x; i < 2 * SLO * SQ / 4; i += ST) d32[i] = s32[i];
  }
  const uint32_t gq = threadIdx.x % (ST / SHL), hl = threadIdx.x / (ST / SHL);
  double acc1[TQ][CB], acc2[TQ][CB];
#pragma unroll
  for (int t = 0; t < TQ; t++)
#pragma unroll
    for (int c = 0; c < CB; c++) acc1[t][c] = acc2[t][c] = 0.0;
  double sH[TQ], cH[TQ], sR[TQ], cR[TQ];
#pragma unroll
  for (int t = 0; t < TQ; t++) {  // sin / cos(q R_h) at the thread's first block, and the rotation by SHL blocks
    const double q = a.qv[(size_t)qt * SQ + split_q(gq, t)];
    xns_math::xns_sincos64_acc(q * ((hb + hl) * a.blk), &sH[t], &cH[t]);
    xns_math::xns_sincos64_acc(q * (SHL * a.blk), &sR[t], &cR[t]);
  }
  const double *cq = c64 + 2 * gq, *sq = c64 + SLO * SQ + 2 * gq;
  const float *cqf = c32 + 2 * gq, *sqf = c32 + SLO * SQ + 2 * gq;
  for (uint32_t s = 0; s < nsteps; s++) {
    cp_async_wait_all();
    __syncthreads();  // step s's rows have landed; every thread is done with the other stage
    if (s + 1 < nsteps) prefetch(s + 1, (s + 1) & 1);
    const uint32_t h = hb + s * SHL + hl;
    if (h < he) {
      double c1[TQ][CB], s1[TQ][CB];
      xns_f2::f2 c2[TQ / 2][CB], s2[TQ / 2][CB];  // FP32 sums, q pairs (2g, 2g + 1), (32 + 2g, 33 + 2g)
#pragma unroll
      for (int t = 0; t < TQ; t++)
#pragma unroll
        for (int c = 0; c < CB; c++) c1[t][c] = s1[t][c] = 0.0;
#pragma unroll
      for (int t = 0; t < TQ / 2; t++)
#pragma unroll
        for (int c = 0; c < CB; c++) c2[t][c] = s2[t][c] = 0ull;
      const double *g1 = gs64 + (s & 1) * G1N + hl * SLO * GS;
      const float *g2 = gs32 + (s & 1) * G1N + hl * SLO * GS;
#pragma unroll 4
      for (int l = 0; l < SLO; l++) {
        const double2 ca = *reinterpret_cast<const double2 *>(cq + l * SQ);
        const double2 cb = *reinterpret_cast<const double2 *>(cq + l * SQ + 32);
        const double2 sa = *reinterpret_cast<const double2 *>(sq + l * SQ);
        const double2 sb = *reinterpret_cast<const double2 *>(sq + l * SQ + 32);
        const double cv[TQ] = {ca.x, ca.y, cb.x, cb.y}, sv[TQ] = {sa.x, sa.y, sb.x, sb.y};
        const xns_f2::f2 cfp[2] = {*reinterpret_cast<const xns_f2::f2 *>(cqf + l * SQ),
                                   *reinterpret_cast<const xns_f2::f2 *>(cqf + l * SQ + 32)};
        const xns_f2::f2 sfp[2] = {*reinterpret_cast<const xns_f2::f2 *>(sqf + l * SQ),
                                   *reinterpret_cast<const xns_f2::f2 *>(sqf + l * SQ + 32)};
        double g[GS];
        float gf[GS];
        if constexpr (GS == 4) {
          const double2 u = *reinterpret_cast<const double2 *>(g1 + l * GS);
          const double2 v = *reinterpret_cast<const double2 *>(g1 + l * GS + 2);
          const float4 w = *reinterpret_cast<const float4 *>(g2 + l * GS);
          g[0] = u.x;
          g[1] = u.y;
          g[2] = v.x;
          g[3] = v.y;
          gf[0] = w.x;
          gf[1] = w.y;
          gf[2] = w.z;
          gf[3] = w.w;
        } else {
#pragma unroll
          for (int c = 0; c < GS; c++) {
            g[c] = g1[l * GS + c];
            gf[c] = g2[l * GS + c];
          }
        }
#pragma unroll
        for (int c = 0; c < CB; c++) {
#pragma unroll
          for (int t = 0; t < TQ; t++) {
            c1[t][c] = __fma_rn(cv[t], g[c], c1[t][c]);
            s1[t][c] = __fma_rn(sv[t], g[c], s1[t][c]);
          }
          const xns_f2::f2 gp = xns_f2::splat(gf[c]);
#pragma unroll
          for (int t = 0; t < TQ / 2; t++) {
            c2[t][c] = xns_f2::fma(cfp[t], gp, c2[t][c]);
            s2[t][c] = xns_f2::fma(sfp[t], gp, s2[t][c]);
          }
        }
      }
#pragma unroll
      for (int t = 0; t < TQ; t++) {
#pragma unroll
        for (int c = 0; c < CB; c++) {
          acc1[t][c] = __fma_rn(sH[t], c1[t][c], __fma_rn(cH[t], s1[t][c], acc1[t][c]));
          const float cc = (t & 1) ? xns_f2::hi(c2[t / 2][c]) : xns_f2::lo(c2[t / 2][c]);
          const float ss = (t & 1) ? xns_f2::hi(s2[t / 2][c]) : xns_f2::lo(s2[t / 2][c]);
          acc2[t][c] = __fma_rn(sH[t], (double)cc, __fma_rn(cH[t], (double)ss, acc2[t][c]));
        }
      }
    }
#pragma unroll
    for (int t = 0; t < TQ; t++) {  // on to the thread's next block, SHL blocks on
      const double sv = sH[t];
      sH[t] = __fma_rn(sv, cR[t], cH[t] * sR[t]);
      cH[t] = __fma_rn(cH[t], cR[t], -(sv * sR[t]));
    }
  }
  // reduce over the 16 block lanes in a fixed order: red[hl][which][c][j]
  __syncthreads();
  double *red = c64;
#pragma unroll
  for (int t = 0; t < TQ; t++)
#pragma unroll
    for (int c = 0; c < CB; c++) {
      const uint32_t j = split_q(gq, t);
      red[((size_t)(hl * 2 + 0) * CB + c) * SQ + j] = acc1[t][c];
      red[((size_t)(hl * 2 + 1) * CB + c) * SQ + j] = acc2[t][c];
    }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < 2 * CB * SQ; i += ST) {  // i = (which * CB + c) * SQ + j
    double sum = 0;
    for (int l = 0; l < SHL; l++) sum += red[(size_t)l * 2 * CB * SQ + i];
    const uint32_t wc = i / SQ, j = i % SQ;
    a.part[((size_t)sp * 2 * CB + wc) * a.nq_pad + (size_t)qt * SQ + j] = sum;
  }
}

// out_G[c0 + c][iq] and out_T[...] = sums of the parts over the splits, in split order.
__global__ void split_reduce_kernel(const double *__restrict__ part, uint32_t nsplit, uint32_t cb, uint32_t nq,
                                    uint32_t nq_pad, uint32_t c0, double *__restrict__ outG, double *__restrict__ outT) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;  // (which, c, iq)
  if (i >= 2 * cb * nq) return;
  const uint32_t iq = i % nq, wc = i / nq, which = wc / cb, c = wc % cb;
  double s = 0;
  for (uint32_t p = 0; p < nsplit; p++) s += part[((size_t)p * 2 * cb + wc) * nq_pad + iq];
  (which ? outT : outG)[(size_t)(c0 + c) * nq + iq] = s;
}

template <int CB>
int launch_split(xns_ctx *ctx, const SplitArgs &a, uint32_t grid) {
  const size_t smem = split_smem_bytes(gstride(CB));
  XNS_CUDA(ctx, cudaFuncSetAttribute(split_sum_kernel<CB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  split_sum_kernel<CB><<<grid, ST, smem, ctx->stream>>>(a);
  return XNS_OK;
}

}  // namespace

// G[c][iq] = sum_k (n_c(k) / r_k) sin(q r_k) and T[c][iq] = sum_k (n_c(k) / r_k^2) sin(q r_k) for the
// ncols histogram columns (column c at d_hist + c * ldh, nh bins).  Scratch: SLOT_SPLIT.
int xns_hist_transform_split(xns_ctx *ctx, const unsigned long long *d_hist, uint32_t ncols, uint32_t nh, size_t ldh,
                             double bin, const double *q, uint32_t nq, double *d_G, double *d_T) {
  if (!ncols || !nq || !nh) return XNS_OK;
  const uint32_t nqt = (nq + SQ - 1) / SQ, nq_pad = nqt * SQ;
  const uint32_t nhi = (nh + SLO - 1) / SLO, nh_pad = nhi * SLO;
  const uint32_t cbmax = std::min<uint32_t>(ncols, CBMAX), gsmax = gstride(cbmax);
  // per CTA about 16 waves over the SMs in all, at least 16 blocks per split
  uint32_t nsplit = std::max<uint32_t>(1, ((uint32_t)ctx->num_sms * 16 + nqt - 1) / nqt);
  nsplit = std::min<uint32_t>(nsplit, std::max<uint32_t>(1, nhi / SHL));
  const uint32_t hps = (nhi + nsplit - 1) / nsplit;
  nsplit = (nhi + hps - 1) / hps;
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t bA64 = up(sizeof(double) * (size_t)nqt * 2 * SLO * SQ), bA32 = up(sizeof(float) * (size_t)nqt * 2 * SLO * SQ);
  const size_t bqv = up(sizeof(double) * nq_pad), bG1 = up(sizeof(double) * (size_t)nh_pad * gsmax);
  const size_t bG2 = up(sizeof(float) * (size_t)nh_pad * gsmax), bpart = up(sizeof(double) * (size_t)nsplit * 2 * cbmax * nq_pad);
  const size_t bq = up(sizeof(double) * nq);
  void *base;
  int st;
  if ((st = xns_scratch(ctx, SLOT_SPLIT, bA64 + bA32 + bqv + bG1 + bG2 + bpart + bq, &base))) return st;
  char *p = (char *)base;
  double *A64 = (double *)p;
  float *A32 = (float *)(p += bA64);
  double *qv = (double *)(p += bA32);
  double *G1 = (double *)(p += bqv);
  float *G2 = (float *)(p += bG1);
  double *part = (double *)(p += bG2);
  double *dqm = (double *)(p += bpart);
  {  // the q values as given (not a fitted uniform mesh)
    void *h;
    if ((st = xns_pinned(ctx, sizeof(double) * nq, &h))) return st;
    XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    memcpy(h, q, sizeof(double) * nq);
    XNS_CUDA(ctx, cudaMemcpyAsync(dqm, h, sizeof(double) * nq, cudaMemcpyHostToDevice, ctx->stream));
  }
  split_tables_kernel<<<(nq_pad * SLO + 255) / 256, 256, 0, ctx->stream>>>(dqm, nq, nq_pad, bin, A64, A32, qv);
  XNS_LAUNCHED(ctx);
  for (uint32_t c0 = 0; c0 < ncols; c0 += CBMAX) {
    const uint32_t cb = std::min<uint32_t>(CBMAX, ncols - c0), gs = gstride(cb);
    split_weights_kernel<<<(nh_pad + 255) / 256, 256, 0, ctx->stream>>>(d_hist, ldh, c0, cb, gs, nh, nh_pad, bin, G1, G2);
    XNS_LAUNCHED(ctx);
    SplitArgs a;
    a.A64 = A64;
    a.A32 = A32;
    a.G1 = G1;
    a.G2 = G2;
    a.qv = qv;
    a.part = part;
    a.nhi = nhi;
    a.nq_pad = nq_pad;
    a.nsplit = nsplit;
    a.hi_per_split = hps;
    a.blk = SLO * bin;
    const uint32_t grid = nqt * nsplit;
    switch (cb) {
      case 1: st = launch_split<1>(ctx, a, grid); break;
      case 2: st = launch_split<2>(ctx, a, grid); break;
      case 3: st = launch_split<3>(ctx, a, grid); break;
      default: st = launch_split<4>(ctx, a, grid); break;
    }
    if (st) return st;
    XNS_LAUNCHED(ctx);
    split_reduce_kernel<<<(2 * cb * nq + 255) / 256, 256, 0, ctx->stream>>>(part, nsplit, cb, nq, nq_pad, c0, d_G, d_T);
    XNS_LAUNCHED(ctx);
  }
  XNS_CUDA(ctx, cudaGetLastError());
  return XNS_OK;
}

// Host-buffer entry: G[c][i] = sum_k hist[c][k] sin(q_i r_k) / (q_i r_k + 1e-8), from the split sums
// (sin(0) / (0 + 1e-8) = 0 at q = 0, as in the reference).
extern "C" int xns_hist_transform_split(xns_ctx *ctx, const uint64_t *hist, uint32_t ncols, uint32_t nh, double bin,
                                        const double *q, uint32_t nq, double *G) {
  if (!ctx) return XNS_ERR_ARG;
  if (!hist || !q || !G || !ncols || !nh || !nq) return xns_fail(ctx, XNS_ERR_ARG, "transform: null or empty argument");
  int st;
  void *dh, *dG;
  if ((st = xns_scratch(ctx, SLOT_HIST, sizeof(uint64_t) * ncols * nh, &dh))) return st;
  if ((st = xns_scratch(ctx, SLOT_TC_OUT, 2 * sizeof(double) * ncols * nq, &dG))) return st;
  XNS_CUDA(ctx, cudaMemcpyAsync(dh, hist, sizeof(uint64_t) * ncols * nh, cudaMemcpyHostToDevice, ctx->stream));
  if ((st = xns_timer_start(ctx))) return st;
  if ((st = xns_stage_begin(ctx, STAGE_IQ))) return st;
  double *dT = (double *)dG + (size_t)ncols * nq;
  if ((st = xns_hist_transform_split(ctx, (const unsigned long long *)dh, ncols, nh, nh, bin, q, nq, (double *)dG, dT)))
    return st;
  if ((st = xns_stage_end(ctx, STAGE_IQ))) return st;
  if ((st = xns_timer_stop(ctx))) return st;
  std::vector<double> both(2 * (size_t)ncols * nq);
  XNS_CUDA(ctx, cudaMemcpyAsync(both.data(), dG, sizeof(double) * both.size(), cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (uint32_t c = 0; c < ncols; c++)
    for (uint32_t i = 0; i < nq; i++) {
      const double g = both[(size_t)c * nq + i], t = both[((size_t)ncols + c) * nq + i];
      G[(size_t)c * nq + i] = q[i] != 0.0 ? g / q[i] - 1e-8 * t / (q[i] * q[i]) : 0.0;
    }
  return XNS_OK;
}
