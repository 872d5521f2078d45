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
// outer weights sin / cos(q R_h) follow h by a rotation.  Per (q, bin, column): two FP64 FMAs, instead
// of a sinc value and its digits per element.  T is summed by sinc_eps_kernel (an FP64 rotation over
// bins) from n / r^2: exactly per bin below EPS_R_FINE, and beyond it in bins of EPS_W (a multiple
// of the bin) with the phase at the bin centre.  Moving a term's phase by at most EPS_W / 2 changes
// eps T / q^2 by at most eps EPS_W / (2 EPS_R_FINE) = 5e-12 of the sum's term magnitudes n / (q r).
//
// split_sum_kernel: a CTA takes 64 q (the tables, 64 KB, in shared memory) and a range of blocks h;
// each thread takes 4 q x CB columns and every 16th block of the range, each step's 16 blocks of
// weights staged in shared memory by cp.async (two stages).  Partial sums per CTA are reduced over the
// CTA's threads in a fixed order and over the h ranges by split_reduce_kernel, so the result does not
// depend on scheduling.
#include <string.h>

#include <algorithm>
#include <vector>

#include "sinc_engine.cuh"
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

// Column stride of the G table: the columns of a pass.
__host__ __device__ constexpr int gstride(int cb) { return cb; }

// Tables per q tile qt: A64[qt][0][l][j] = cos(q r_l), A64[qt][1][l][j] = sin(q r_l) for q the tile's
// j-th value (0 past nq); qv the padded mesh.
__global__ void split_tables_kernel(const double *__restrict__ qmesh, uint32_t nq, uint32_t nq_pad,
                                    double bin, double *__restrict__ A64, double *__restrict__ qv) {
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
}

// G1[k][c] = n_c(k) / r_k for the columns c0 .. c0 + cb - 1 of this pass, zero past nh.
__global__ void split_weights_kernel(const unsigned long long *__restrict__ hist, size_t ldh, uint32_t c0, uint32_t cb,
                                     uint32_t nh, uint32_t nh_pad, double bin, double *__restrict__ G1) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nh_pad) return;
  const double r = (k + 0.5) * bin;
  for (uint32_t c = 0; c < cb; c++) {
    const double n = k < nh ? (double)hist[(size_t)(c0 + c) * ldh + k] : 0.0;
    G1[(size_t)k * cb + c] = n / r;
  }
}

// The +1e-8 histograms: H[c][b] = sum of n_c(k) / r_k^2 over the bins k of [b ratio, (b + 1) ratio)
// that lie in [k_lo, k_hi), for every column.
constexpr double EPS_R_FINE = 20.0;  // A: T per bin below this distance
constexpr double EPS_W = 0.02;       // A: T in bins of at least this width beyond it
__global__ void split_eps_hist_kernel(const unsigned long long *__restrict__ hist, size_t ldh, uint32_t ncols, uint32_t k_lo,
                                      uint32_t k_hi, double bin, uint32_t ratio, uint32_t nb, double *__restrict__ H) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;  // (c, b)
  if (i >= ncols * nb) return;
  const uint32_t c = i / nb, b = i % nb;
  double s = 0;
  for (uint32_t k = max(k_lo, b * ratio); k < min(k_hi, (b + 1) * ratio); k++) {
    const double r = (k + 0.5) * bin;
    s += (double)hist[(size_t)c * ldh + k] / (r * r);
  }
  H[i] = s;
}

struct SplitArgs {
  const double *A64;
  const double *G1;
  const double *qv;
  double *part;  // [split][CB][nq_pad]
  uint32_t nhi, nq_pad, nsplit, hi_per_split;
  double blk;  // 64 bin
};

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Shared memory of split_sum_kernel: the q tile's tables (FP64 cos, sin: 64 KB), then two stages of
// one step's G rows (16 blocks x 64 bins x GS columns): 112 KB at three columns, two CTAs per SM.
__host__ __device__ constexpr size_t split_stage_bytes(int gs) { return (size_t)SHL * SLO * gs * 8; }
__host__ __device__ constexpr size_t split_smem_bytes(int gs) {
  return (size_t)2 * SLO * SQ * 8 + 2 * split_stage_bytes(gs);
}

// A thread's q: 2g, 2g + 1, 32 + 2g, 33 + 2g of the tile (g = thread % 16), so that the 16 threads of a
// half warp read 256 contiguous bytes per table load.
__device__ __forceinline__ uint32_t split_q(uint32_t g, int t) { return (t < 2 ? 0u : 32u) + 2 * g + (t & 1); }

template <int CB>
__global__ void __launch_bounds__(ST, 2) split_sum_kernel(SplitArgs a) {
  constexpr int GS = gstride(CB);
  constexpr uint32_t G1N = SHL * SLO * GS;  // doubles of one step's G rows
  extern __shared__ __align__(16) unsigned char smem[];
  double *c64 = reinterpret_cast<double *>(smem);  // [SLO][SQ] cos, then [SLO][SQ] sin
  double *gs64 = c64 + 2 * SLO * SQ;               // [stage][G1N]
  const uint32_t qt = blockIdx.x / a.nsplit, sp = blockIdx.x % a.nsplit;
  const uint32_t hb = sp * a.hi_per_split, he = min(hb + a.hi_per_split, a.nhi);
  const uint32_t nsteps = (he - hb + SHL - 1) / SHL;
  // one step's G rows: blocks hb + SHL s .. + SHL - 1 are contiguous in the table; blocks past the
  // last one are not copied (their threads do not read them)
  auto prefetch = [&](uint32_t s, uint32_t stage) {
    const uint32_t h0 = hb + s * SHL, nrow = min((uint32_t)SHL, a.nhi - h0);
    const uint32_t n1 = nrow * SLO * GS / 2;  // 16-byte pieces
    const double *g1 = a.G1 + (size_t)h0 * SLO * GS;
    double *d1 = gs64 + stage * G1N;
    for (uint32_t i = threadIdx.x; i < n1; i += ST) cp_async16(d1 + 2 * i, g1 + 2 * i);
    cp_async_commit();
  };
  if (nsteps) prefetch(0, 0);
  {  // the tile's tables
    const double2 *src = reinterpret_cast<const double2 *>(a.A64 + (size_t)qt * 2 * SLO * SQ);
    double2 *dst = reinterpret_cast<double2 *>(c64);
    for (uint32_t i = threadIdx.x; i < 2 * SLO * SQ / 2; i += ST) dst[i] = src[i];
  }
  const uint32_t gq = threadIdx.x % (ST / SHL), hl = threadIdx.x / (ST / SHL);
  double acc[TQ][CB];
#pragma unroll
  for (int t = 0; t < TQ; t++)
#pragma unroll
    for (int c = 0; c < CB; c++) acc[t][c] = 0.0;
  double sH[TQ], cH[TQ], sR[TQ], cR[TQ];
#pragma unroll
  for (int t = 0; t < TQ; t++) {  // sin / cos(q R_h) at the thread's first block, and the rotation by SHL blocks
    const double q = a.qv[(size_t)qt * SQ + split_q(gq, t)];
    xns_math::xns_sincos64_acc(q * ((hb + hl) * a.blk), &sH[t], &cH[t]);
    xns_math::xns_sincos64_acc(q * (SHL * a.blk), &sR[t], &cR[t]);
  }
  const double *cq = c64 + 2 * gq, *sq = c64 + SLO * SQ + 2 * gq;
  for (uint32_t s = 0; s < nsteps; s++) {
    cp_async_wait_all();
    __syncthreads();  // step s's rows have landed; every thread is done with the other stage
    if (s + 1 < nsteps) prefetch(s + 1, (s + 1) & 1);
    const uint32_t h = hb + s * SHL + hl;
    if (h < he) {
      double c1[TQ][CB], s1[TQ][CB];
#pragma unroll
      for (int t = 0; t < TQ; t++)
#pragma unroll
        for (int c = 0; c < CB; c++) c1[t][c] = s1[t][c] = 0.0;
      const double *g1 = gs64 + (s & 1) * G1N + hl * SLO * GS;
#pragma unroll 4
      for (int l = 0; l < SLO; l++) {
        const double2 ca = *reinterpret_cast<const double2 *>(cq + l * SQ);
        const double2 cb = *reinterpret_cast<const double2 *>(cq + l * SQ + 32);
        const double2 sa = *reinterpret_cast<const double2 *>(sq + l * SQ);
        const double2 sb = *reinterpret_cast<const double2 *>(sq + l * SQ + 32);
        const double cv[TQ] = {ca.x, ca.y, cb.x, cb.y}, sv[TQ] = {sa.x, sa.y, sb.x, sb.y};
        double g[CB];
#pragma unroll
        for (int c = 0; c < CB; c++) g[c] = g1[l * GS + c];
#pragma unroll
        for (int c = 0; c < CB; c++)
#pragma unroll
          for (int t = 0; t < TQ; t++) {
            c1[t][c] = __fma_rn(cv[t], g[c], c1[t][c]);
            s1[t][c] = __fma_rn(sv[t], g[c], s1[t][c]);
          }
      }
#pragma unroll
      for (int t = 0; t < TQ; t++)
#pragma unroll
        for (int c = 0; c < CB; c++) acc[t][c] = __fma_rn(sH[t], c1[t][c], __fma_rn(cH[t], s1[t][c], acc[t][c]));
    }
#pragma unroll
    for (int t = 0; t < TQ; t++) {  // on to the thread's next block, SHL blocks on
      const double sv = sH[t];
      sH[t] = __fma_rn(sv, cR[t], cH[t] * sR[t]);
      cH[t] = __fma_rn(cH[t], cR[t], -(sv * sR[t]));
    }
  }
  // reduce over the 16 block lanes in a fixed order: red[hl][c][j]
  __syncthreads();
  double *red = c64;
#pragma unroll
  for (int t = 0; t < TQ; t++)
#pragma unroll
    for (int c = 0; c < CB; c++) red[((size_t)hl * CB + c) * SQ + split_q(gq, t)] = acc[t][c];
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < CB * SQ; i += ST) {  // i = c * SQ + j
    double sum = 0;
    for (int l = 0; l < SHL; l++) sum += red[(size_t)l * CB * SQ + i];
    const uint32_t c = i / SQ, j = i % SQ;
    a.part[((size_t)sp * CB + c) * a.nq_pad + (size_t)qt * SQ + j] = sum;
  }
}

// out_G[c0 + c][iq] = sum of the parts over the splits, in split order.
__global__ void split_reduce_kernel(const double *__restrict__ part, uint32_t nsplit, uint32_t cb, uint32_t nq,
                                    uint32_t nq_pad, uint32_t c0, double *__restrict__ outG) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;  // (c, iq)
  if (i >= cb * nq) return;
  const uint32_t iq = i % nq, c = i / nq;
  double s = 0;
  for (uint32_t p = 0; p < nsplit; p++) s += part[((size_t)p * cb + c) * nq_pad + iq];
  outG[(size_t)(c0 + c) * nq + iq] = s;
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
  // the +1e-8 histograms: per bin below k_fine (EPS_R_FINE), in bins of ratio bins (EPS_W) above it
  const uint32_t ratio = std::max<uint32_t>(1, (uint32_t)std::ceil(EPS_W / bin - 1e-9));
  const uint32_t neps = (nh + ratio - 1) / ratio;
  const uint32_t k_fine = std::min(nh, std::min(neps * ratio, ((uint32_t)std::ceil(EPS_R_FINE / bin) + ratio - 1) / ratio * ratio));
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t bA64 = up(sizeof(double) * (size_t)nqt * 2 * SLO * SQ), bqv = up(sizeof(double) * nq_pad);
  const size_t bG1 = up(sizeof(double) * (size_t)nh_pad * gsmax), bpart = up(sizeof(double) * (size_t)nsplit * cbmax * nq_pad);
  const size_t bq = up(sizeof(double) * nq), beps = up(sizeof(double) * (size_t)ncols * neps);
  const size_t bfine = up(sizeof(double) * (size_t)ncols * std::max<uint32_t>(k_fine, 1));
  void *base;
  int st;
  if ((st = xns_scratch(ctx, SLOT_SPLIT, bA64 + bqv + bG1 + bpart + bq + beps + bfine, &base))) return st;
  char *p = (char *)base;
  double *A64 = (double *)p;
  double *qv = (double *)(p += bA64);
  double *G1 = (double *)(p += bqv);
  double *part = (double *)(p += bG1);
  double *dqm = (double *)(p += bpart);
  double *heps = (double *)(p += bq);
  double *hfine = (double *)(p += beps);
  {  // the q values as given (not a fitted uniform mesh)
    void *h;
    if ((st = xns_pinned(ctx, sizeof(double) * nq, &h))) return st;
    XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    memcpy(h, q, sizeof(double) * nq);
    XNS_CUDA(ctx, cudaMemcpyAsync(dqm, h, sizeof(double) * nq, cudaMemcpyHostToDevice, ctx->stream));
  }
  split_tables_kernel<<<(nq_pad * SLO + 255) / 256, 256, 0, ctx->stream>>>(dqm, nq, nq_pad, bin, A64, qv);
  XNS_LAUNCHED(ctx);
  for (uint32_t c0 = 0; c0 < ncols; c0 += CBMAX) {
    const uint32_t cb = std::min<uint32_t>(CBMAX, ncols - c0);
    split_weights_kernel<<<(nh_pad + 255) / 256, 256, 0, ctx->stream>>>(d_hist + (size_t)c0 * ldh, ldh, 0, cb, nh, nh_pad,
                                                                        bin, G1);
    XNS_LAUNCHED(ctx);
    SplitArgs a;
    a.A64 = A64;
    a.G1 = G1;
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
    split_reduce_kernel<<<(cb * nq + 255) / 256, 256, 0, ctx->stream>>>(part, nsplit, cb, nq, nq_pad, c0, d_G);
    XNS_LAUNCHED(ctx);
  }
  // T (sinc_eps_kernel adds into a zeroed T): per bin below k_fine, in the coarse bins above it
  XNS_CUDA(ctx, cudaMemsetAsync(d_T, 0, sizeof(double) * ncols * nq, ctx->stream));
  if (k_fine) {
    split_eps_hist_kernel<<<(ncols * k_fine + 255) / 256, 256, 0, ctx->stream>>>(d_hist, ldh, ncols, 0, k_fine, bin, 1,
                                                                               k_fine, hfine);
    XNS_LAUNCHED(ctx);
    dim3 eg((nq + 127) / 128, (k_fine + xns_sinc::EPS_RUN - 1) / xns_sinc::EPS_RUN, ncols);
    xns_sinc::sinc_eps_kernel<<<eg, 128, 0, ctx->stream>>>(hfine, k_fine, bin, 0.0, 0.0, dqm, nq, d_T);
    XNS_LAUNCHED(ctx);
  }
  if (k_fine < nh) {
    split_eps_hist_kernel<<<(ncols * neps + 255) / 256, 256, 0, ctx->stream>>>(d_hist, ldh, ncols, k_fine, nh, bin, ratio,
                                                                             neps, heps);
    XNS_LAUNCHED(ctx);
    // (the coarse bins below k_fine hold nothing)
    dim3 eg((nq + 127) / 128, (neps + xns_sinc::EPS_RUN - 1) / xns_sinc::EPS_RUN, ncols);
    xns_sinc::sinc_eps_kernel<<<eg, 128, 0, ctx->stream>>>(heps, neps, ratio * bin, 0.0, 0.0, dqm, nq, d_T);
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
