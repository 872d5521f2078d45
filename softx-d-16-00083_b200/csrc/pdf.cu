// PDF / RDF / rPDF from the pair-distance histogram (replaces the PDF branch of calcPDFandDebye,
// CalcFunctions.cpp:919-960, and calcPartialRDF/PDF/RPDFkernel + calcPDFkernel,
// CalcFunctionsCUDA.cu:1048-1075).
//
// One thread per bin computes every element pair's partial value and the weighted total, with the
// reference's operations in the reference's order (explicitly rounded FP64, no contraction), so the
// result is bit-identical to the reference's.  The per-pair constants (mult, sub, SL_a SL_b/<SL>^2)
// are formed on the host with the reference's expressions.  As in the reference, pair t's radius at
// bin k is (t*nhist + k + 0.5)*bin: the loop variable there runs over the concatenated histogram
// (:939-951), which is the bin centre for the first element pair only.
#include <string.h>

#include "xns_internal.cuh"

namespace {

struct PdfPair {
  double mult, sub, mij;
};

__global__ void pdf_kernel(const unsigned long long *__restrict__ hist, uint32_t nhist, uint32_t P, double bin, int pdftype,
                           const PdfPair *__restrict__ pp, double *__restrict__ pdf) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nhist) return;
  double total = 0.0;
  for (uint32_t t = 0; t < P; t++) {
    const uint32_t i = t * nhist + k;  // the reference's loop index (unsigned int)
    const double h = (double)hist[i];
    double v;
    if (pdftype == XNS_RDF) {
      v = __dmul_rn(h, pp[t].mult);
    } else {
      const double r = __dmul_rn(__dadd_rn((double)i, 0.5), bin);
      if (pdftype == XNS_PDF) v = __ddiv_rn(__dmul_rn(h, pp[t].mult), __dmul_rn(r, r));
      else v = __dsub_rn(__ddiv_rn(__dmul_rn(h, pp[t].mult), r), __dmul_rn(pp[t].sub, r));
    }
    pdf[(size_t)nhist + i] = v;
    total = __dadd_rn(total, __dmul_rn(v, pp[t].mij));
  }
  pdf[k] = total;
}

}  // namespace

int xns_pdf_device(xns_ctx *ctx, const unsigned long long *d_hist, const uint32_t *n_el, uint32_t nel, uint32_t nhist,
                   double bin, int pdftype, double p0, const double *sl, double *d_pdf) {
  if (pdftype != XNS_RDF && pdftype != XNS_PDF && pdftype != XNS_RPDF)
    return xns_fail(ctx, XNS_ERR_ARG, "PDF type must be XNS_RDF, XNS_PDF or XNS_RPDF");
  if (!sl) return xns_fail(ctx, XNS_ERR_ARG, "PDF needs the per-element weights (sl)");
  const uint32_t P = xns_npairs(nel);
  unsigned int ntot = 0;
  for (uint32_t e = 0; e < nel; e++) ntot += n_el[e];
  // CalcFunctions.cpp:925-930
  double fav2 = 0;
  for (uint32_t e = 0; e < nel; e++) fav2 += sl[e] * n_el[e];
  fav2 /= ntot;
  fav2 *= fav2;
  std::vector<PdfPair> pp;
  for (uint32_t a = 0; a < nel; a++)
    for (uint32_t b = a; b < nel; b++) {
      PdfPair x;
      x.mij = sl[a] * sl[b] / fav2;  // :933
      x.sub = 0;
      switch (pdftype) {            // :934-953
        case XNS_RDF: x.mult = 2. / (bin * ntot); break;
        case XNS_PDF: x.mult = 0.5 / (XNS_PI * bin * p0 * ntot); break;
        default:
          x.mult = 2. / (bin * ntot);
          x.sub = (b > a) ? 8. * XNS_PI * p0 * double(n_el[a]) * double(n_el[b]) / ((double(ntot)) * (double(ntot)))
                          : 4. * XNS_PI * p0 * ((double(n_el[a])) * (double(n_el[a]))) / ((double(ntot)) * (double(ntot)));
      }
      pp.push_back(x);
    }
  void *d, *h;
  int st;
  if ((st = xns_scratch(ctx, SLOT_AUX, sizeof(PdfPair) * P, &d))) return st;
  if ((st = xns_pinned(ctx, sizeof(PdfPair) * P, &h))) return st;
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  memcpy(h, pp.data(), sizeof(PdfPair) * P);
  XNS_CUDA(ctx, cudaMemcpyAsync(d, h, sizeof(PdfPair) * P, cudaMemcpyHostToDevice, ctx->stream));
  if ((st = xns_stage_begin(ctx, STAGE_PDF))) return st;
  pdf_kernel<<<(nhist + 255) / 256, 256, 0, ctx->stream>>>(d_hist, nhist, P, bin, pdftype, (const PdfPair *)d, d_pdf);
  XNS_LAUNCHED(ctx);
  if ((st = xns_stage_end(ctx, STAGE_PDF))) return st;
  // the AUX slot is reused by later stages: make sure this kernel has read it
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XNS_OK;
}

extern "C" int xns_calc_pdf(xns_ctx *ctx, const uint64_t *hist, const uint32_t *n_el, uint32_t nel, uint32_t nhist, double bin,
                            int pdftype, double p0, const double *sl, double *pdf) {
  if (!ctx) return XNS_ERR_ARG;
  if (!hist || !n_el || !pdf || nel == 0 || nhist == 0) return xns_fail(ctx, XNS_ERR_ARG, "PDF: null pointer or zero size");
  const uint32_t P = xns_npairs(nel);
  const size_t hbytes = sizeof(uint64_t) * (size_t)P * nhist, pbytes = sizeof(double) * (size_t)(1 + P) * nhist;
  void *d_hist, *d_pdf;
  int st;
  if ((st = xns_scratch(ctx, SLOT_HIST, hbytes, &d_hist))) return st;
  if ((st = xns_scratch(ctx, SLOT_OUT2, pbytes, &d_pdf))) return st;
  XNS_CUDA(ctx, cudaMemcpyAsync(d_hist, hist, hbytes, cudaMemcpyHostToDevice, ctx->stream));
  if ((st = xns_timer_start(ctx))) return st;
  if ((st = xns_pdf_device(ctx, (const unsigned long long *)d_hist, n_el, nel, nhist, bin, pdftype, p0, sl, (double *)d_pdf)))
    return st;
  if ((st = xns_timer_stop(ctx))) return st;
  XNS_CUDA(ctx, cudaMemcpyAsync(pdf, d_pdf, pbytes, cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XNS_OK;
}
