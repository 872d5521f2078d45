#include <string.h>

#include "sinc_engine.cuh"

namespace xns_sinc {

__global__ void sinc_epilogue_kernel(const double *__restrict__ partial, int grid, uint32_t ncls, uint32_t nel,
                                     uint32_t nparts, uint32_t nblocks, const uint32_t *__restrict__ pair_a,
                                     const uint32_t *__restrict__ pair_b, const double *__restrict__ w,
                                     const uint32_t *__restrict__ n_el_block, double q0, double dq,
                                     const double *__restrict__ qmesh, uint32_t nq, uint32_t ntot, int polar, double lambda,
                                     int over_q, int self_term, const double *__restrict__ eps_t, double *__restrict__ out) {
  const uint32_t iq = blockIdx.x * blockDim.x + threadIdx.x;
  if (iq >= nq) return;
  const uint32_t P = nel * (nel + 1) / 2;
  const double q = qmesh ? qmesh[iq] : q0 + iq * dq;
  double fac = 1.0;
  if (polar) {  // PolarFactor1D, CalcFunctions.cpp:460-468
    double st = q * (lambda * 0.25 / XNS_PI), c2 = 1. - 2. * st * st;
    fac = 0.5 * (1. + c2 * c2);
  }
  double total = 0;
  uint32_t part = 0;
  for (uint32_t u = 0; u < nblocks; u++)
    for (uint32_t v = u; v < nblocks; v++, part++) {
      double I = 0;
      for (uint32_t t = 0; t < P; t++) {
        const uint32_t c = part * P + t;
        double S = 0;
        for (int g = 0; g < grid; g++) S += partial[((size_t)g * ncls + c) * nq + iq];
        if (over_q) {  // sin(0)/(0 + 1e-8) = 0 in the reference
          S = (q != 0.0) ? S / q : 0.0;
          if (eps_t && q != 0.0) S -= SINC_EPS * eps_t[(size_t)c * nq + iq] / (q * q);
        }
        I += S * w[(size_t)pair_a[t] * nq + iq] * w[(size_t)pair_b[t] * nq + iq] * 2.;
      }
      if (u == v && self_term)
        for (uint32_t e = 0; e < nel; e++) {
          double we = w[(size_t)e * nq + iq];
          I += n_el_block[e * nblocks + u] * (we * we);
        }
      I = I / ntot * fac;
      total += I;
      if (nparts > 1) out[(size_t)(1 + part) * nq + iq] = I;
    }
  out[iq] = total;
}

__global__ void sinc_eps_kernel(const double *__restrict__ H, uint32_t nb, double bin, double q0, double dq,
                                const double *__restrict__ qmesh, uint32_t nq, double *__restrict__ T) {
  const uint32_t iq = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t b0 = blockIdx.y * EPS_RUN, b1 = min(nb, b0 + EPS_RUN);
  const double *h = H + (size_t)blockIdx.z * nb;
  if (iq >= nq) return;
  const double q = qmesh ? qmesh[iq] : q0 + iq * dq;
  double sr, cr, sw, cw;
  xns_math::xns_sincos64(q * (((double)b0 + 0.5) * bin), &sr, &cr);
  xns_math::xns_sincos64(q * bin, &sw, &cw);
  double acc = 0.0;
  for (uint32_t b = b0; b < b1; b++) {
    acc = __fma_rn(h[b], sr, acc);
    const double s2 = __fma_rn(sr, cw, cr * sw);
    cr = __fma_rn(cr, cw, -sr * sw);
    sr = s2;
  }
  atomicAdd(T + (size_t)blockIdx.z * nq + iq, acc);
}

size_t sinc_smem_bytes(int M, int lanes_per_slot, size_t stage_bytes) {
  (void)lanes_per_slot;  // one FP64 column per thread whatever the slot width
  return sizeof(double) * M * SE_THREADS + sizeof(PairRec) * SE_TILE + stage_bytes;
}

int sinc_upload_q(xns_ctx *ctx, const double *q, uint32_t nq, const double **d_q) {
  void *d, *h;
  int st;
  if ((st = xns_scratch(ctx, SLOT_QMESH, sizeof(double) * nq, &d))) return st;
  if ((st = xns_pinned(ctx, sizeof(double) * nq, &h))) return st;
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  memcpy(h, q, sizeof(double) * nq);
  XNS_CUDA(ctx, cudaMemcpyAsync(d, h, sizeof(double) * nq, cudaMemcpyHostToDevice, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *d_q = (const double *)d;
  return XNS_OK;
}

int sinc_epilogue(xns_ctx *ctx, int grid, uint32_t ncls, uint32_t nel, uint32_t nblocks, const uint32_t *n_el_block,
                  const double *q, uint32_t nq, bool uniform, double q0, double dq, const double *d_w, uint32_t ntot,
                  int polar, double lambda, double *d_out, const double *partial, bool over_q, bool self_term,
                  const double *eps_t) {
  const uint32_t P = xns_npairs(nel);
  const size_t nu32 = 2 * (size_t)P + (size_t)nel * nblocks;
  void *aux, *h;
  int st;
  if ((st = xns_scratch(ctx, SLOT_AUX, sizeof(uint32_t) * nu32, &aux))) return st;
  if ((st = xns_pinned(ctx, sizeof(uint32_t) * nu32, &h))) return st;
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  uint32_t *hu = (uint32_t *)h;
  uint32_t t = 0;
  for (uint32_t a = 0; a < nel; a++)
    for (uint32_t b = a; b < nel; b++, t++) {
      hu[t] = a;
      hu[P + t] = b;
    }
  memcpy(hu + 2 * P, n_el_block, sizeof(uint32_t) * nel * nblocks);
  XNS_CUDA(ctx, cudaMemcpyAsync(aux, h, sizeof(uint32_t) * nu32, cudaMemcpyHostToDevice, ctx->stream));
  const double *d_q = nullptr;
  if (!uniform && (st = sinc_upload_q(ctx, q, nq, &d_q))) return st;
  const uint32_t *d_pa = (const uint32_t *)aux;
  const uint32_t nparts = nblocks * (nblocks + 1) / 2;
  if (!partial) partial = (const double *)ctx->slot_ptr[SLOT_PARTIAL];
  sinc_epilogue_kernel<<<(nq + 127) / 128, 128, 0, ctx->stream>>>(partial, grid, ncls,
                                                                  nel, nparts, nblocks, d_pa, d_pa + P, d_w, d_pa + 2 * P,
                                                                  q0, dq, d_q, nq, ntot, polar, lambda, over_q, self_term,
                                                                  eps_t, d_out);
  XNS_LAUNCHED(ctx);
  return XNS_OK;
}

}  // namespace xns_sinc
