// Histogram -> I(q) (replaces calcInt1DHist, CalcFunctions.cpp:810-911, and calcIntHistKernel*,
// CalcFunctionsCUDA.cu:923-1045) and the fused histogram + PDF + I(q) entry point (calcPDFandDebye,
// CalcFunctions.cpp:912-968).
//
//   I(q) = [ sum_e N_e w_e^2 + 2 sum_{a<=b} w_a w_b sum_k n_ab(k) sin(q r_k)/(q r_k + 1e-8) ] / N,
//   r_k = (k + 0.5) * bin; empty bins contribute nothing (the reference skips them, :857).
//
// The contraction over bins runs in FP64 by angle splitting (hist_split.cu): at the deep low-q minima
// of I(q) the bin sum cancels to 1e-5..1e-6 of its terms, and FP32 sums leave 3e-5..5e-5 of I(q)
// there.  The transform yields sum_k (n(k) / r_k) sin(q r_k) and the first-order +1e-8 sum; the shared
// epilogue (sinc_engine.cu) divides by q, subtracts 1e-8 T / q^2 and applies the weights, the self
// term, 1/N and the polarisation factor.
#include <string.h>

#include "sinc_engine.cuh"
#include "tc_gemm.cuh"

using namespace xns_sinc;

int xns_hist_iq_device(xns_ctx *ctx, const unsigned long long *d_hist, const uint32_t *n_el, uint32_t nel, uint32_t nhist,
                       double bin, const double *q, uint32_t nq, const double *d_w, int polar, double lambda, double *d_I) {
  const uint32_t P = xns_npairs(nel);
  uint32_t ntot = 0;
  for (uint32_t e = 0; e < nel; e++) ntot += n_el[e];
  if (ntot == 0) return xns_fail(ctx, XNS_ERR_ARG, "I(q): no atoms");
  double q0 = 0, dq = 0;
  const bool uniform = xns_uniform_mesh(q, nq, &q0, &dq);
  int st;
  void *d_G, *d_T;
  if ((st = xns_scratch(ctx, SLOT_PARTIAL, sizeof(double) * P * nq, &d_G))) return st;
  if ((st = xns_scratch(ctx, SLOT_EPS_T, sizeof(double) * P * nq, &d_T))) return st;
  if ((st = xns_stage_begin(ctx, STAGE_IQ))) return st;
  if ((st = xns_hist_transform_split(ctx, d_hist, P, nhist, nhist, bin, q, nq, (double *)d_G, (double *)d_T))) return st;
  if ((st = sinc_epilogue(ctx, 1, P, nel, 1, n_el, q, nq, uniform, q0, dq, d_w, ntot, polar, lambda, d_I,
                          (const double *)d_G, true, true, (const double *)d_T)))
    return st;
  return xns_stage_end(ctx, STAGE_IQ);
}

extern "C" int xns_calc_int_1d_hist(xns_ctx *ctx, const uint64_t *hist, const uint32_t *n_el, uint32_t nel, uint32_t nhist,
                                    double bin, const double *q, uint32_t nq, int source, const double *const *ff,
                                    const double *sl, int polar, double lambda, double *I) {
  if (!ctx) return XNS_ERR_ARG;
  if (!hist || !n_el || !q || !I || nel == 0 || nq == 0 || nhist == 0 || !(bin > 0))
    return xns_fail(ctx, XNS_ERR_ARG, "I(q) from histogram: null pointer or zero size");
  int st;
  const size_t hbytes = sizeof(uint64_t) * (size_t)xns_npairs(nel) * nhist;
  void *d_hist, *d_I;
  if ((st = xns_scratch(ctx, SLOT_HIST, hbytes, &d_hist))) return st;
  XNS_CUDA(ctx, cudaMemcpyAsync(d_hist, hist, hbytes, cudaMemcpyHostToDevice, ctx->stream));
  double *d_w;
  if ((st = xns_upload_weights(ctx, nel, nq, source, ff, sl, &d_w))) return st;
  if ((st = xns_scratch(ctx, SLOT_OUT, sizeof(double) * nq, &d_I))) return st;
  if ((st = xns_timer_start(ctx))) return st;
  if ((st = xns_hist_iq_device(ctx, (const unsigned long long *)d_hist, n_el, nel, nhist, bin, q, nq, d_w, polar, lambda,
                               (double *)d_I)))
    return st;
  if ((st = xns_timer_stop(ctx))) return st;
  XNS_CUDA(ctx, cudaMemcpyAsync(I, d_I, sizeof(double) * nq, cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XNS_OK;
}

extern "C" int xns_pdf_and_debye_device(xns_ctx *ctx, const double *xyz_dev, const uint32_t *n_el, uint32_t nel,
                                        uint32_t nhist, double bin, int scenario, int pdftype, double p0, const double *q,
                                        uint32_t nq, int source, const double *const *ff, const double *sl, int polar,
                                        double lambda, double *I_dev, double *pdf_dev, uint64_t *hist_dev) {
  if (!ctx) return XNS_ERR_ARG;
  if (scenario != XNS_DEBYE_HIST && scenario != XNS_PDF_ONLY && scenario != XNS_DEBYE_PDF)
    return xns_fail(ctx, XNS_ERR_ARG, "scenario must be Debye_hist (2), PDFonly (3) or DebyePDF (4)");
  const bool want_iq = scenario != XNS_PDF_ONLY, want_pdf = scenario != XNS_DEBYE_HIST;
  if (!hist_dev || (want_iq && (!I_dev || !q || nq == 0)) || (want_pdf && (!pdf_dev || !sl)))
    return xns_fail(ctx, XNS_ERR_ARG, "pdf_and_debye_device: missing output or weights for the scenario");
  int st;
  DevCoords dc;
  if ((st = xns_coords_from_device(ctx, xyz_dev, n_el, nel, &dc))) return st;
  if (dc.ntot == 0) return xns_fail(ctx, XNS_ERR_ARG, "pdf_and_debye_device: no atoms");
  double *d_w = nullptr;
  if (want_iq && (st = xns_upload_weights(ctx, nel, nq, source, ff, sl, &d_w))) return st;
  if ((st = xns_timer_start(ctx))) return st;
  if ((st = xns_hist_device(ctx, dc, nhist, bin, (unsigned long long *)hist_dev))) return st;
  if (want_pdf &&
      (st = xns_pdf_device(ctx, (const unsigned long long *)hist_dev, n_el, nel, nhist, bin, pdftype, p0, sl, pdf_dev)))
    return st;
  if (want_iq && (st = xns_hist_iq_device(ctx, (const unsigned long long *)hist_dev, n_el, nel, nhist, bin, q, nq, d_w,
                                          polar, lambda, I_dev)))
    return st;
  return xns_timer_stop(ctx);
}

extern "C" int xns_pdf_and_debye_from_hist_device(xns_ctx *ctx, const uint64_t *hist_dev, const uint32_t *n_el, uint32_t nel,
                                                  uint32_t nhist, double bin, int scenario, int pdftype, double p0,
                                                  const double *q, uint32_t nq, int source, const double *const *ff,
                                                  const double *sl, int polar, double lambda, double *I_dev,
                                                  double *pdf_dev) {
  if (!ctx) return XNS_ERR_ARG;
  if (scenario != XNS_DEBYE_HIST && scenario != XNS_PDF_ONLY && scenario != XNS_DEBYE_PDF)
    return xns_fail(ctx, XNS_ERR_ARG, "scenario must be Debye_hist (2), PDFonly (3) or DebyePDF (4)");
  const bool want_iq = scenario != XNS_PDF_ONLY, want_pdf = scenario != XNS_DEBYE_HIST;
  if (!hist_dev || !n_el || nel == 0 || (want_iq && (!I_dev || !q || nq == 0)) || (want_pdf && (!pdf_dev || !sl)))
    return xns_fail(ctx, XNS_ERR_ARG, "pdf_and_debye_from_hist_device: missing input, output or weights");
  int st;
  double *d_w = nullptr;
  if (want_iq && (st = xns_upload_weights(ctx, nel, nq, source, ff, sl, &d_w))) return st;
  if ((st = xns_timer_start(ctx))) return st;
  if (want_pdf &&
      (st = xns_pdf_device(ctx, (const unsigned long long *)hist_dev, n_el, nel, nhist, bin, pdftype, p0, sl, pdf_dev)))
    return st;
  if (want_iq && (st = xns_hist_iq_device(ctx, (const unsigned long long *)hist_dev, n_el, nel, nhist, bin, q, nq, d_w,
                                          polar, lambda, I_dev)))
    return st;
  return xns_timer_stop(ctx);
}

extern "C" int xns_calc_pdf_and_debye(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel,
                                      uint32_t nhist, double bin, int scenario, int pdftype, double p0, const double *q,
                                      uint32_t nq, int source, const double *const *ff, const double *sl, int polar,
                                      double lambda, double *I, double *pdf, uint64_t *hist_out) {
  if (!ctx) return XNS_ERR_ARG;
  if (scenario != XNS_DEBYE_HIST && scenario != XNS_PDF_ONLY && scenario != XNS_DEBYE_PDF)
    return xns_fail(ctx, XNS_ERR_ARG, "scenario must be Debye_hist (2), PDFonly (3) or DebyePDF (4)");
  const bool want_iq = scenario != XNS_PDF_ONLY, want_pdf = scenario != XNS_DEBYE_HIST;
  if ((want_iq && (!I || !q || nq == 0)) || (want_pdf && (!pdf || !sl)))
    return xns_fail(ctx, XNS_ERR_ARG, "calc_pdf_and_debye: missing output or weights for the scenario");
  int st;
  DevCoords dc;
  if ((st = xns_upload_coords(ctx, xyz_el, n_el, nel, &dc))) return st;
  if (dc.ntot == 0) return xns_fail(ctx, XNS_ERR_ARG, "calc_pdf_and_debye: no atoms");
  const uint32_t P = xns_npairs(nel);
  const size_t hbytes = sizeof(uint64_t) * (size_t)P * nhist;
  void *d_hist, *d_I = nullptr, *d_pdf = nullptr;
  double *d_w = nullptr;
  if ((st = xns_scratch(ctx, SLOT_HIST, hbytes, &d_hist))) return st;
  if (want_iq) {
    if ((st = xns_upload_weights(ctx, nel, nq, source, ff, sl, &d_w))) return st;
    if ((st = xns_scratch(ctx, SLOT_OUT, sizeof(double) * nq, &d_I))) return st;
  }
  if (want_pdf && (st = xns_scratch(ctx, SLOT_OUT2, sizeof(double) * (size_t)(1 + P) * nhist, &d_pdf))) return st;
  if ((st = xns_timer_start(ctx))) return st;
  if ((st = xns_hist_device(ctx, dc, nhist, bin, (unsigned long long *)d_hist))) return st;
  if (want_pdf &&
      (st = xns_pdf_device(ctx, (const unsigned long long *)d_hist, n_el, nel, nhist, bin, pdftype, p0, sl, (double *)d_pdf)))
    return st;
  if (want_iq && (st = xns_hist_iq_device(ctx, (const unsigned long long *)d_hist, n_el, nel, nhist, bin, q, nq, d_w, polar,
                                          lambda, (double *)d_I)))
    return st;
  if ((st = xns_timer_stop(ctx))) return st;
  if (want_iq) XNS_CUDA(ctx, cudaMemcpyAsync(I, d_I, sizeof(double) * nq, cudaMemcpyDeviceToHost, ctx->stream));
  if (want_pdf)
    XNS_CUDA(ctx, cudaMemcpyAsync(pdf, d_pdf, sizeof(double) * (size_t)(1 + P) * nhist, cudaMemcpyDeviceToHost, ctx->stream));
  if (hist_out) XNS_CUDA(ctx, cudaMemcpyAsync(hist_out, d_hist, hbytes, cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XNS_OK;
}
