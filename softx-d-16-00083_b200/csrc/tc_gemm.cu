// Split-BF16 sinc transform on tcgen05 (see tc_gemm.cuh for the algorithm and operand layout).
//
// One CTA per SM (192 KB of shared memory: two stages of {Sh, Sl, Hh, Hl} tiles), 6 warps:
//   warp 0, one thread: loads, one cp.async.bulk per tile into the stage's mbarrier;
//   warp 1, one thread: issues 12 tcgen05.mma (3 products x 4 K16 steps) per stage into a
//                       128 x BN FP32 accumulator in tensor memory, commits to free the stage;
//   warps 2-5:          read the accumulator (tcgen05.ld, 32 lanes each) when a (column tile, q tile)
//                       segment ends and add it into the FP64 output.
// The (column tile, q tile, k tile) work units are split evenly over the CTAs in that order
// (stream-K): a CTA's range covers parts of one or two output tiles.  Every wait is bounded by a
// 2 s wall-clock limit; on expiry the CTA raises an error flag, lets its copies and MMAs drain and
// releases its tensor memory before returning.
#include <algorithm>

#include "tc_gemm.cuh"
#include "tc_ptx.cuh"
#include "xmath.cuh"

using namespace xns_tc;
using namespace xns_ptx;

namespace {

__global__ void __launch_bounds__(THREADS, 1) sinc_gemm_kernel(const GemmArgs g) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) unsigned long long bars[2 * STAGES + 3];
  __shared__ uint32_t tmem_sh;
  __shared__ int abort_sh;
  const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
  const uint32_t full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[STAGES]);
  const uint32_t tfull = smem_u32(&bars[2 * STAGES]), tempty = smem_u32(&bars[2 * STAGES + 1]);
  const uint32_t drain = smem_u32(&bars[2 * STAGES + 2]);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  volatile int *abort = &abort_sh;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    mbar_init(tfull, 1);
    mbar_init(tempty, 4 * 32);
    mbar_init(drain, 1);
    abort_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_sh)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_sh;

  const unsigned long long KT = g.KT;
  const unsigned long long units = (unsigned long long)g.NT * g.MT * KT;
  const unsigned long long u0 = units * blockIdx.x / gridDim.x, u1 = units * (blockIdx.x + 1) / gridDim.x;
  const uint32_t btile = g.BN * BK * 2;

  if (warp == 0) {
    if (lane == 0) {  // loader
      uint32_t fills[STAGES] = {};
      unsigned long long i = 0;
      for (unsigned long long u = u0; u < u1; ++u, ++i) {
        const uint32_t s = (uint32_t)(i % STAGES), k = (uint32_t)(i / STAGES);
        if (k > 0 && !mbar_wait(empty0 + 8 * s, (k - 1) & 1u, abort, WAIT_LIMIT_NS)) {
          abort_sh = 1;
          atomicOr(g.err, 1);
          break;
        }
        const uint32_t kt = (uint32_t)(u % KT);
        const unsigned long long r = u / KT;
        const uint32_t mt = (uint32_t)(r % g.MT), nt = (uint32_t)(r / g.MT);
        const uint32_t dst = base + s * STAGE_BYTES, bar = full0 + 8 * s;
        const size_t ao = ((size_t)mt * g.KT + kt) * A_TILE, bo = ((size_t)nt * g.KT + kt) * btile;
        mbar_expect_tx(bar, 2u * A_TILE + 2u * btile);
        bulk_g2s(dst, g.Ah + ao, A_TILE, bar);
        bulk_g2s(dst + A_TILE, g.Al + ao, A_TILE, bar);
        bulk_g2s(dst + 2 * A_TILE, g.Bh + bo, btile, bar);
        bulk_g2s(dst + 2 * A_TILE + B_TILE_MAX, g.Bl + bo, btile, bar);
        fills[s] = k + 1;
      }
      if (*abort)  // the copies already issued land before this CTA's shared memory is released
        for (int s = 0; s < STAGES; s++)
          if (fills[s]) mbar_wait(full0 + 8 * s, (fills[s] - 1) & 1u, nullptr, DRAIN_LIMIT_NS);
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((g.BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
      uint32_t seg = 0;
      bool issued = false;
      unsigned long long i = 0;
      for (unsigned long long u = u0; u < u1; ++u, ++i) {
        const uint32_t s = (uint32_t)(i % STAGES), k = (uint32_t)(i / STAGES);
        const bool first = (u == u0) || (u % KT == 0);
        const bool last = (u + 1 == u1) || ((u + 1) % KT == 0);
        if (first && seg > 0) {
          if (!mbar_wait(tempty, (seg - 1) & 1u, abort, WAIT_LIMIT_NS)) {
            abort_sh = 1;
            atomicOr(g.err, 1);
            break;
          }
          tc_fence_after();
        }
        if (!mbar_wait(full0 + 8 * s, k & 1u, abort, WAIT_LIMIT_NS)) {
          abort_sh = 1;
          atomicOr(g.err, 1);
          break;
        }
        tc_fence_after();
        const uint32_t a_h = base + s * STAGE_BYTES, a_l = a_h + A_TILE;
        const uint32_t b_h = a_h + 2 * A_TILE, b_l = b_h + B_TILE_MAX;
#pragma unroll
        for (int j = 0; j < BK / 16; j++) {
          const uint32_t off = j * 32;  // 16 BF16 along K inside the 128-byte swizzle row
          tc_mma(tmem, sw128_desc(a_h + off), sw128_desc(b_h + off), idesc, (first && j == 0) ? 0u : 1u);
          tc_mma(tmem, sw128_desc(a_h + off), sw128_desc(b_l + off), idesc, 1u);
          tc_mma(tmem, sw128_desc(a_l + off), sw128_desc(b_h + off), idesc, 1u);
        }
        issued = true;
        tc_commit(empty0 + 8 * s);
        if (last) {
          tc_commit(tfull);
          seg++;
        }
      }
      if (*abort && issued) {  // MMAs in flight finish before the tensor memory is released
        tc_commit(drain);
        mbar_wait(drain, 0, nullptr, DRAIN_LIMIT_NS);
      }
    }
  } else {  // accumulator drain: warp w reads TMEM lanes 32*(w%4) .. +31
    const uint32_t wq = warp & 3;
    uint32_t seg = 0;
    for (unsigned long long us = u0; us < u1; seg++) {
      const unsigned long long r = us / KT, ue = (r + 1) * KT < u1 ? (r + 1) * KT : u1;
      const uint32_t mt = (uint32_t)(r % g.MT), nt = (uint32_t)(r / g.MT);
      const bool ok = mbar_wait(tfull, seg & 1u, abort, WAIT_LIMIT_NS);
      if (__any_sync(0xffffffffu, !ok)) {
        abort_sh = 1;
        if (lane == 0) atomicOr(g.err, 1);
        break;
      }
      tc_fence_after();
      const uint32_t m = mt * BM + wq * 32 + lane;
      for (uint32_t c = 0; c < g.BN; c += 16) {
        float v[16];
        tc_ld16(tmem + ((wq * 32u) << 16) + c, v);
        if (m < g.m_valid) {
#pragma unroll
          for (int j = 0; j < 16; j++) {
            const uint32_t n = nt * g.BN + c + j;
            if (n < g.n_valid) atomicAdd(g.out + (size_t)n * g.ldo + m, (double)v[j]);
          }
        }
      }
      tc_fence_before();
      mbar_arrive(tempty);
      us = ue;
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16 *hi, __nv_bfloat16 *lo) {
  *hi = __float2bfloat16_rn(x);
  *lo = __float2bfloat16_rn(x - __bfloat162float(*hi));
}

__device__ __forceinline__ void store_chunk(uint8_t *dst_h, uint8_t *dst_l, const float *v) {
  __align__(16) __nv_bfloat16 h[8], l[8];
#pragma unroll
  for (int i = 0; i < 8; i++) split_bf16(v[i], &h[i], &l[i]);
  *(uint4 *)dst_h = *(const uint4 *)h;
  *(uint4 *)dst_l = *(const uint4 *)l;
}

// One CTA per (mt, kt) tile; a thread writes 8 consecutive k of one row (one 16-byte chunk).
__global__ void pack_sinc_kernel(const double *__restrict__ q, uint32_t nq, double bin, uint32_t nh, uint32_t KT,
                                 uint8_t *__restrict__ Ah, uint8_t *__restrict__ Al) {
  const uint32_t tile = blockIdx.x, mt = tile / KT, kt = tile % KT;
  uint8_t *th = Ah + (size_t)tile * A_TILE, *tl = Al + (size_t)tile * A_TILE;
  for (uint32_t c = threadIdx.x; c < BM * (BK / 8); c += blockDim.x) {
    const uint32_t row = c >> 3, ch = c & 7, m = mt * BM + row, k0 = kt * BK + ch * 8;
    float v[8];
    const double qm = m < nq ? q[m] : 0.0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const uint32_t k = k0 + i;
      float s = 0.f;
      if (m < nq && k < nh) {
        const double x = qm * ((k + 0.5) * bin);  // reference bin centre (CalcFunctions.cpp:858)
        s = x > 0 ? xns_math::xns_sin(x) / (float)x : 1.f;
      }
      v[i] = s;
    }
    const uint32_t off = sw128_offset(row, ch * 8);
    store_chunk(th + off, tl + off, v);
  }
}

// One CTA per (nt, kt) tile of BN rows (columns of the histogram matrix).
__global__ void pack_counts_kernel(const unsigned long long *__restrict__ hist, uint32_t ncols, uint32_t nh, size_t ldh,
                                   uint32_t BN, uint32_t KT, uint8_t *__restrict__ Bh, uint8_t *__restrict__ Bl) {
  const uint32_t tile = blockIdx.x, nt = tile / KT, kt = tile % KT;
  const size_t bt = (size_t)BN * BK * 2;
  uint8_t *th = Bh + (size_t)tile * bt, *tl = Bl + (size_t)tile * bt;
  for (uint32_t c = threadIdx.x; c < BN * (BK / 8); c += blockDim.x) {
    const uint32_t row = c >> 3, ch = c & 7, n = nt * BN + row, k0 = kt * BK + ch * 8;
    float v[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const uint32_t k = k0 + i;
      v[i] = (n < ncols && k < nh) ? (float)hist[(size_t)n * ldh + k] : 0.f;
    }
    const uint32_t off = sw128_offset(row, ch * 8);
    store_chunk(th + off, tl + off, v);
  }
}

}  // namespace

int xns_tc_pack_sinc(xns_ctx *ctx, const double *d_q, uint32_t nq, double bin, uint32_t nh, uint32_t MT, uint32_t KT,
                     uint8_t *Ah, uint8_t *Al) {
  pack_sinc_kernel<<<MT * KT, 256, 0, ctx->stream>>>(d_q, nq, bin, nh, KT, Ah, Al);
  XNS_LAUNCHED(ctx);
  return XNS_OK;
}

int xns_tc_pack_counts(xns_ctx *ctx, const unsigned long long *d_hist, uint32_t ncols, uint32_t nh, size_t ldh,
                       uint32_t BN, uint32_t NT, uint32_t KT, uint8_t *Bh, uint8_t *Bl) {
  pack_counts_kernel<<<NT * KT, 256, 0, ctx->stream>>>(d_hist, ncols, nh, ldh, BN, KT, Bh, Bl);
  XNS_LAUNCHED(ctx);
  return XNS_OK;
}

int xns_tc_sinc_gemm(xns_ctx *ctx, const GemmArgs &g, int grid) {
  static bool attr_set[XNS_MAX_DEVICES] = {};  // the attribute is per device; set once on each
  if (ctx->device < 0 || ctx->device >= XNS_MAX_DEVICES || !attr_set[ctx->device]) {
    XNS_CUDA(ctx, cudaFuncSetAttribute(sinc_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
    if (ctx->device >= 0 && ctx->device < XNS_MAX_DEVICES) attr_set[ctx->device] = true;
  }
  if (g.BN < 16 || g.BN > BN_MAX || g.BN % 16) return xns_fail(ctx, XNS_ERR_ARG, "sinc GEMM: column tile not in 16..256");
  const unsigned long long units = (unsigned long long)g.NT * g.MT * g.KT;
  if (units == 0) return XNS_OK;
  if (grid <= 0) grid = ctx->num_sms;
  grid = (int)std::min<unsigned long long>((unsigned long long)grid, units);
  sinc_gemm_kernel<<<grid, THREADS, SMEM_BYTES, ctx->stream>>>(g);
  XNS_LAUNCHED(ctx);
  return XNS_OK;
}

int xns_tc_hist_transform(xns_ctx *ctx, const unsigned long long *d_hist, uint32_t ncols, uint32_t nh, size_t ldh,
                          double bin, const double *q, uint32_t nq, double *d_G) {
  if (!ncols || !nq) return XNS_OK;
  const uint32_t MT = (nq + BM - 1) / BM, KT = (nh + BK - 1) / BK;
  const uint32_t BN = std::min<uint32_t>(BN_MAX, (ncols + 15) / 16 * 16), NT = (ncols + BN - 1) / BN;
  int st;
  // sinc planes: rebuilt only when the q mesh, the bin width or the K extent change
  const size_t a_plane = (size_t)MT * KT * A_TILE;
  void *A;
  const bool same = ctx->tc_bin == bin && ctx->tc_kt == KT && ctx->tc_q.size() == nq &&
                    std::equal(q, q + nq, ctx->tc_q.begin()) && ctx->slot_size[SLOT_TC_A] >= 2 * a_plane;
  if ((st = xns_scratch(ctx, SLOT_TC_A, 2 * a_plane, &A))) return st;
  if (!same) {
    void *dq;
    if ((st = xns_scratch(ctx, SLOT_QMESH, sizeof(double) * nq, &dq))) return st;
    XNS_CUDA(ctx, cudaMemcpyAsync(dq, q, sizeof(double) * nq, cudaMemcpyHostToDevice, ctx->stream));
    if ((st = xns_tc_pack_sinc(ctx, (const double *)dq, nq, bin, nh, MT, KT, (uint8_t *)A, (uint8_t *)A + a_plane)))
      return st;
    ctx->tc_q.assign(q, q + nq);
    ctx->tc_bin = bin;
    ctx->tc_kt = KT;
  }
  const size_t b_plane = (size_t)NT * KT * BN * BK * 2;
  void *B;
  if ((st = xns_scratch(ctx, SLOT_TC_B, 2 * b_plane, &B))) return st;
  if ((st = xns_tc_pack_counts(ctx, d_hist, ncols, nh, ldh, BN, NT, KT, (uint8_t *)B, (uint8_t *)B + b_plane))) return st;
  void *flags;
  if ((st = xns_scratch(ctx, SLOT_FLAGS, 64, &flags))) return st;
  XNS_CUDA(ctx, cudaMemsetAsync(flags, 0, sizeof(int), ctx->stream));
  XNS_CUDA(ctx, cudaMemsetAsync(d_G, 0, sizeof(double) * ncols * nq, ctx->stream));
  GemmArgs g{};
  g.Ah = (const uint8_t *)A;
  g.Al = (const uint8_t *)A + a_plane;
  g.Bh = (const uint8_t *)B;
  g.Bl = (const uint8_t *)B + b_plane;
  g.MT = MT;
  g.NT = NT;
  g.KT = KT;
  g.BN = BN;
  g.out = d_G;
  g.ldo = nq;
  g.m_valid = nq;
  g.n_valid = ncols;
  g.err = (int *)flags;
  if ((st = xns_tc_sinc_gemm(ctx, g, 0))) return st;
  int err = 0;
  XNS_CUDA(ctx, cudaMemcpyAsync(&err, flags, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (err) return xns_fail(ctx, XNS_ERR_CUDA, "sinc GEMM: a pipeline wait ran out of time");
  return XNS_OK;
}

// Histogram columns (host, ncols x nh u64, column-major by histogram) -> G (host, ncols x nq) on the
// tensor cores.  A test and measurement entry for the split-BF16 transform itself.
extern "C" int xns_hist_transform_bf16x3(xns_ctx *ctx, const uint64_t *hist, uint32_t ncols, uint32_t nh, double bin,
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
  if ((st = xns_tc_hist_transform(ctx, (const unsigned long long *)dh, ncols, nh, nh, bin, q, nq, (double *)dG))) return st;
  if ((st = xns_stage_end(ctx, STAGE_IQ))) return st;
  if ((st = xns_timer_stop(ctx))) return st;
  XNS_CUDA(ctx, cudaMemcpyAsync(G, dG, sizeof(double) * ncols * nq, cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XNS_OK;
}
