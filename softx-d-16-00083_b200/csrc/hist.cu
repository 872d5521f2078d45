// Pair-distance histogram (replaces calcHist, CalcFunctions.cpp:757-809, and calcHistKernel,
// CalcFunctionsCUDA.cu:814-844).
//
// Counts must be bit-identical to the reference, which bins (unsigned int)(rij / bin) with
// rij = sqrt((dx*dx + dy*dy) + dz*dz) evaluated in IEEE FP64 without FMA (typedefs.h:130, g++ -O3 on
// x86-64).  The kernel therefore forms d2 with explicitly rounded FP64 operations, then decides the
// bin from d2 with a cheap estimate that is exact whenever it is not within a proven margin of a
// bin edge, and with the reference's own correctly rounded sqrt and divide otherwise (see ref_bin).
#include <math.h>

#include <algorithm>

#include "schedule.cuh"

namespace {

constexpr int HIST_TILE = 256;  // atoms per tile on both sides = threads per CTA

// Float with the exponent and top 20 mantissa bits of d (d in [2^-126, 2^128)), built with integer
// operations only: the estimate needs no conversion-pipe instruction.
__device__ __forceinline__ float trunc_to_float(double d) {
  int hi = __double2hiint(d);
  return __int_as_float((hi - (896 << 20)) << 3);
}

__device__ __forceinline__ double float_to_double_exact(float f) {
  int b = __float_as_int(f);
  return __hiloint2double((b >> 3) + (896 << 20), b << 29);
}

// Reference bin index (unsigned)(fl(fl(sqrt(d2)) / bin)), or 0xffffffff when it is >= nhist.
//
// Estimate: f = d2 truncated to float (rel. err < 2^-20), y = rsqrtf(f) (max error 2 ulp, CUDA
// Programming Guide), so y = (1 + e)/sqrt(d2) with |e| < 0.75*2^-20.  One Newton step in FP64,
// r1 = r0 + (d2 - r0^2) * y/2 with r0 = d2*y, leaves |r1/sqrt(d2) - 1| < 2^-39.8, and
// t = r1 * fl(1/bin) is within t*2^-39.7 of the reference quotient Q = fl(fl(sqrt(d2))/bin)
// (itself within 2^-52 of sqrt(d2)/bin).  With t < nhist, any |t - round(t)| >= margin =
// nhist*2^-37 proves floor(Q) = floor(t); otherwise the exact IEEE operations decide.
__device__ __forceinline__ uint32_t ref_bin(double d2, double bin, double inv_bin, double margin, uint32_t nhist) {
  const double MAGIC = 6755399441055744.0;  // 1.5 * 2^52: adding it rounds to an integer in the low word
  int hi = __double2hiint(d2);
  if (hi >= (897 << 20) && hi < (1151 << 20)) {
    float y = rsqrtf(trunc_to_float(d2));
    double yd = float_to_double_exact(y);
    double r0 = __dmul_rn(d2, yd);
    double res = __fma_rn(-r0, r0, d2);
    double r1 = __fma_rn(res, 0.5 * yd, r0);
    double t = __dmul_rn(r1, inv_bin);
    if (t < (double)nhist - 1.0) {
      double u = __dadd_rn(t, MAGIC);
      double v = __dsub_rn(u, MAGIC);
      double d = __dsub_rn(t, v);
      if (fabs(d) >= margin) return (uint32_t)__double2loint(u) - (d < 0.0 ? 1u : 0u);
    }
  }
  double q = __ddiv_rn(__dsqrt_rn(d2), bin);
  if (!(q < (double)nhist)) return 0xffffffffu;
  return (uint32_t)q;
}

__device__ __forceinline__ double ref_dist2(double xi, double yi, double zi, double xj, double yj, double zj) {
  double dx = __dsub_rn(xi, xj), dy = __dsub_rn(yi, yj), dz = __dsub_rn(zi, zj);
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

__global__ void __launch_bounds__(HIST_TILE) hist_tiles_kernel(const double *__restrict__ X, const double *__restrict__ Y,
                                                               const double *__restrict__ Z, const SegPair *__restrict__ sp,
                                                               int nsp, unsigned long long ntiles, double bin, double inv_bin,
                                                               double margin, uint32_t nhist,
                                                               unsigned long long *__restrict__ hist,
                                                               unsigned int *__restrict__ n_out_of_range) {
  __shared__ double sx[HIST_TILE], sy[HIST_TILE], sz[HIST_TILE];
  const int tid = threadIdx.x;
  unsigned int bad = 0;
  for (unsigned long long w = blockIdx.x; w < ntiles; w += gridDim.x) {
    int s;
    uint32_t I, J;
    xns_decode_tile(sp, nsp, w, &s, &I, &J);
    const SegPair p = sp[s];
    const uint32_t ia = I * HIST_TILE + tid;
    const uint32_t jb = J * HIST_TILE;
    const uint32_t nj = min((uint32_t)HIST_TILE, p.nb - jb);
    if (tid < (int)nj) {
      sx[tid] = X[p.b0 + jb + tid];
      sy[tid] = Y[p.b0 + jb + tid];
      sz[tid] = Z[p.b0 + jb + tid];
    }
    __syncthreads();
    if (ia < p.na) {
      const double xi = X[p.a0 + ia], yi = Y[p.a0 + ia], zi = Z[p.a0 + ia];
      unsigned long long *h = hist + (size_t)p.cls * nhist;
      const uint32_t j0 = (p.same && I == J) ? (uint32_t)tid + 1 : 0u;
      for (uint32_t j = j0; j < nj; j++) {
        double d2 = ref_dist2(xi, yi, zi, sx[j], sy[j], sz[j]);
        uint32_t k = ref_bin(d2, bin, inv_bin, margin, nhist);
        if (k < nhist) atomicAdd(h + k, 1ull);
        else bad++;
      }
    }
    __syncthreads();
  }
  if (bad) atomicAdd(n_out_of_range, bad);
}

}  // namespace

int xns_hist_device(xns_ctx *ctx, const DevCoords &dc, uint32_t nhist, double bin, unsigned long long *d_hist) {
  const uint32_t nel = (uint32_t)dc.n_el.size();
  if (nhist == 0 || !(bin > 0)) return xns_fail(ctx, XNS_ERR_ARG, "histogram: nhist == 0 or bin <= 0");
  const uint32_t P = xns_npairs(nel);
  std::vector<Segment> sa, sb;
  std::vector<uint32_t> cls, same;
  uint32_t t = 0;
  for (uint32_t a = 0; a < nel; a++)
    for (uint32_t b = a; b < nel; b++, t++) {
      sa.push_back({dc.off_el[a], dc.n_el[a]});
      sb.push_back({dc.off_el[b], dc.n_el[b]});
      cls.push_back(t);
      same.push_back(a == b);
    }
  std::vector<SegPair> sched;
  unsigned long long ntiles = xns_build_schedule(sa, sb, cls, same, HIST_TILE, HIST_TILE, &sched);
  int st;
  XNS_CUDA(ctx, cudaMemsetAsync(d_hist, 0, sizeof(unsigned long long) * (size_t)P * nhist, ctx->stream));
  void *flags;
  if ((st = xns_scratch(ctx, SLOT_FLAGS, 64, &flags))) return st;
  XNS_CUDA(ctx, cudaMemsetAsync(flags, 0, 64, ctx->stream));
  if (ntiles == 0) return XNS_OK;
  SegPair *d_sp;
  if ((st = xns_upload_schedule(ctx, sched, &d_sp))) return st;
  int per_sm = 0;
  XNS_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hist_tiles_kernel, HIST_TILE, 0));
  unsigned long long grid = std::min<unsigned long long>(ntiles, (unsigned long long)ctx->num_sms * std::max(per_sm, 1));
  const double margin = (double)nhist * ldexp(1.0, -37);
  if ((st = xns_stage_begin(ctx, STAGE_HIST))) return st;
  hist_tiles_kernel<<<(unsigned)grid, HIST_TILE, 0, ctx->stream>>>(dc.x, dc.y, dc.z, d_sp, (int)sched.size(), ntiles, bin,
                                                                   1.0 / bin, margin, nhist, d_hist, (unsigned int *)flags);
  XNS_LAUNCHED(ctx);
  if ((st = xns_stage_end(ctx, STAGE_HIST))) return st;
  unsigned int bad = 0;
  XNS_CUDA(ctx, cudaMemcpyAsync(&bad, flags, sizeof(bad), cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (bad) return xns_fail(ctx, XNS_ERR_RANGE, "histogram: " + std::to_string(bad) + " pair distances fall beyond nhist bins");
  return XNS_OK;
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
