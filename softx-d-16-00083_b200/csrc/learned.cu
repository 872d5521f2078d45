// Kernels of the learned binning correction (no reference counterpart; xns_b200/learned.py drives
// them together with the perceptron of mlp.cu).
//
// A coarse histogram puts every pair of bin k at its centre r_k.  Expanding sin(q r)/(q r) about r_k to
// second order in the offset d = r - r_k gives, per bin, a correction in the first two moments of d:
//
//   I(q) = s0 [1 + sum_k h_k S(q r_k)] + s0 sum_k h_k [mu1_k D S'(r_k) + m2_k D^2/2 S''(r_k)]
//   S = sin(q r)/(q r),  S' = cos(q r)/r - sin(q r)/(q r^2),
//   S'' = -q sin(q r)/r - 2 cos(q r)/r^2 + 2 sin(q r)/(q r^3)
//
// with h the weighted histogram normalised by N s0, D the bin width, mu1_k = E[d/D] and m2_k = E[(d/D)^2]
// within bin k.  The perceptron predicts (mu1, m2) per bin from the bin's neighbourhood (features below);
// binning_correction_kernel evaluates the second sum.
#include <math.h>

#include "xmath.cuh"
#include "xns_internal.cuh"

namespace {

constexpr int NB = 4;  // neighbours on each side
constexpr int NFEAT = 2 * NB + 1 + 2 * NB + 1;

// Per bin k: log(1 + h_{k+j}) for j = -NB..NB, min(h_{k+j} / (h_k + 1e-12), 16) for j != 0, and the bin
// position k / nh.  Bins outside the histogram count as empty.
__global__ void features_kernel(const double *__restrict__ h, uint32_t nh, float *__restrict__ X) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nh; k += gridDim.x * blockDim.x) {
    float *x = X + (size_t)k * NFEAT;
    const double hk = h[k];
    int f = 0;
    for (int j = -NB; j <= NB; j++) {
      const long kk = (long)k + j;
      x[f++] = (float)log1p(kk >= 0 && kk < nh ? h[kk] : 0.0);
    }
    for (int j = -NB; j <= NB; j++) {
      if (!j) continue;
      const long kk = (long)k + j;
      const double v = kk >= 0 && kk < nh ? h[kk] : 0.0;
      x[f++] = (float)fmin(v / (hk + 1e-12), 16.0);
    }
    x[f++] = (float)k / (float)nh;
  }
}

// dI[iq] = s0 sum_k h_k [mu1_k D S'(q r_k) + m2_k D^2/2 S''(q r_k)], r_k = (k + 0.5) D; FP64 per term.
__global__ void binning_correction_kernel(const double *__restrict__ h, const float *__restrict__ mu, uint32_t nh,
                                          double bin, const double *__restrict__ q, uint32_t nq, double s0,
                                          double *__restrict__ dI) {
  const uint32_t iq = blockIdx.x * blockDim.x + threadIdx.x;
  if (iq >= nq) return;
  const double qq = q[iq];
  double acc = 0.0;
  for (uint32_t k = 0; k < nh; k++) {
    const double hk = h[k];
    if (hk == 0.0) continue;
    const double r = (k + 0.5) * bin, x = qq * r;
    double s, c;
    sincos(x, &s, &c);
    const double ir = 1.0 / r;
    const double d1 = c * ir - s / (qq * r * r);
    const double d2 = -qq * s * ir - 2.0 * c * ir * ir + 2.0 * s / (qq * r * r * r);
    acc += hk * ((double)mu[2 * k] * bin * d1 + 0.5 * (double)mu[2 * k + 1] * bin * bin * d2);
  }
  dI[iq] = s0 * acc;
}

}  // namespace

extern "C" {

int xns_binning_features(xns_ctx *ctx, const double *h, uint32_t nh, float *X) {
  if (!ctx) return XNS_ERR_ARG;
  if (!h || !X || nh == 0) return xns_fail(ctx, XNS_ERR_ARG, "binning features: null pointer or nh == 0");
  int st;
  void *dh, *dX;
  if ((st = xns_scratch(ctx, SLOT_AUX, sizeof(double) * nh, &dh))) return st;
  if ((st = xns_scratch(ctx, SLOT_OUT2, sizeof(float) * nh * NFEAT, &dX))) return st;
  XNS_CUDA(ctx, cudaMemcpyAsync(dh, h, sizeof(double) * nh, cudaMemcpyHostToDevice, ctx->stream));
  features_kernel<<<(nh + 255) / 256, 256, 0, ctx->stream>>>((const double *)dh, nh, (float *)dX);
  XNS_LAUNCHED(ctx);
  XNS_CUDA(ctx, cudaMemcpyAsync(X, dX, sizeof(float) * nh * NFEAT, cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XNS_OK;
}

int xns_binning_correction(xns_ctx *ctx, const double *h, const float *mu, uint32_t nh, double bin, const double *q,
                           uint32_t nq, double s0, double *dI) {
  if (!ctx) return XNS_ERR_ARG;
  if (!h || !mu || !q || !dI || nh == 0 || nq == 0 || !(bin > 0))
    return xns_fail(ctx, XNS_ERR_ARG, "binning correction: null pointer or zero size");
  int st;
  void *dh, *dmu, *dq, *dout;
  if ((st = xns_scratch(ctx, SLOT_AUX, sizeof(double) * nh, &dh))) return st;
  if ((st = xns_scratch(ctx, SLOT_OUT2, sizeof(float) * 2 * nh, &dmu))) return st;
  if ((st = xns_scratch(ctx, SLOT_QMESH, sizeof(double) * nq, &dq))) return st;
  if ((st = xns_scratch(ctx, SLOT_OUT, sizeof(double) * nq, &dout))) return st;
  XNS_CUDA(ctx, cudaMemcpyAsync(dh, h, sizeof(double) * nh, cudaMemcpyHostToDevice, ctx->stream));
  XNS_CUDA(ctx, cudaMemcpyAsync(dmu, mu, sizeof(float) * 2 * nh, cudaMemcpyHostToDevice, ctx->stream));
  XNS_CUDA(ctx, cudaMemcpyAsync(dq, q, sizeof(double) * nq, cudaMemcpyHostToDevice, ctx->stream));
  binning_correction_kernel<<<(nq + 127) / 128, 128, 0, ctx->stream>>>((const double *)dh, (const float *)dmu, nh, bin,
                                                                       (const double *)dq, nq, s0, (double *)dout);
  XNS_LAUNCHED(ctx);
  XNS_CUDA(ctx, cudaMemcpyAsync(dI, dout, sizeof(double) * nq, cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XNS_OK;
}

}  // extern "C"
