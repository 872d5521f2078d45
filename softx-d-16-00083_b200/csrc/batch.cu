// Batched ensembles: the Debye-histogram I(q) of many independent structures in one pass.
//
// The reference evaluates one structure per run (calcPDFandDebye with scenario Debye_hist,
// CalcFunctions.cpp:912-968 over calcHist :757-809 and calcInt1DHist :810-911).  An ensemble
// (disorder or size-distribution averaging) is many such runs; here it is one pipeline:
//   1. one plan for all structures (hist.cu: spatial sort, tile pairs, runs of one class each);
//   2. one persistent histogram launch whose CTAs take runs of any structure from a shared queue,
//      largest first, so that structures of uneven size balance across the SMs;
//   3. one exact tensor-core transform over all (structure, element pair) histogram columns
//      (tc_exact.cu);
//   4. an epilogue that applies each structure's weights, self term, 1/N and polarisation factor.
// Steps 2-4 are memsets and kernels only: xns_batch_create captures them in a CUDA graph once, and
// xns_batch_run replays it.  An optional autotuner times the histogram launch for a few plans
// (spatial cell size, window depth) on the ensemble itself and keeps the fastest.
//
// A batch owns a private context (its own stream and working memory), so it stays valid while the
// caller's context runs other calls.
#include <string.h>

#include <algorithm>

#include "hist_set.cuh"
#include "tc_gemm.cuh"

namespace {

struct StructInfo {
  uint32_t cls_base, e0, nel, ntot;
};

// I[s][iq] = [sum_e N_e w_e^2 + 2 sum_{a<=b} w_a w_b G[cls][iq]] / N_s, times the polarisation factor
// (CalcFunctions.cpp:872-906; PolarFactor1D :460-468).
__global__ void batch_epilogue_kernel(const double *__restrict__ G, const double *__restrict__ w,
                                      const uint32_t *__restrict__ n_el, const StructInfo *__restrict__ si,
                                      const double *__restrict__ q, uint32_t nq, int polar, double lambda,
                                      double *__restrict__ I) {
  const uint32_t iq = blockIdx.x * blockDim.x + threadIdx.x, s = blockIdx.y;
  if (iq >= nq) return;
  const StructInfo S = si[s];
  double acc = 0;
  uint32_t t = S.cls_base;
  for (uint32_t a = 0; a < S.nel; a++) {
    const double wa = w[(size_t)(S.e0 + a) * nq + iq];
    acc += n_el[S.e0 + a] * (wa * wa);
    for (uint32_t b = a; b < S.nel; b++, t++) acc += 2.0 * wa * w[(size_t)(S.e0 + b) * nq + iq] * G[(size_t)t * nq + iq];
  }
  double fac = 1.0;
  if (polar) {
    const double st = q[iq] * (lambda * 0.25 / XNS_PI), c2 = 1. - 2. * st * st;
    fac = 0.5 * (1. + c2 * c2);
  }
  I[(size_t)s * nq + iq] = S.ntot ? acc / S.ntot * fac : 0.0;
}

}  // namespace

struct xns_batch {
  xns_ctx *ctx = nullptr;  // private context
  uint32_t nstruct = 0, nq = 0, nhist = 0, classes = 0;
  HistLaunch hl;
  ExactLaunch xl;
  unsigned long long *d_hist = nullptr;
  double *d_G = nullptr, *d_w = nullptr, *d_I = nullptr, *d_q = nullptr;
  uint32_t *d_nel = nullptr;
  StructInfo *d_si = nullptr;
  int polar = 0;
  double lambda = 0;
  HistTuning tune;
  double tuned_ms = -1;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

int batch_epilogue(xns_batch *b) {
  dim3 grid((b->nq + 127) / 128, b->nstruct);
  batch_epilogue_kernel<<<grid, 128, 0, b->ctx->stream>>>(b->d_G, b->d_w, b->d_nel, b->d_si, b->d_q, b->nq, b->polar,
                                                          b->lambda, b->d_I);
  XNS_LAUNCHED(b->ctx);
  return XNS_OK;
}

// The replayable part: histogram launches, transform launches, epilogue.
int batch_enqueue(xns_batch *b) {
  int st;
  if ((st = xns_hist_enqueue(b->ctx, b->hl))) return st;
  if ((st = xns_tc_exact_enqueue(b->ctx, b->xl))) return st;
  return batch_epilogue(b);
}

int batch_check(xns_batch *b) {
  int st;
  if ((st = xns_hist_check(b->ctx, b->hl))) return st;
  return xns_tc_exact_check(b->ctx, b->xl);
}

// Plans the ensemble: uploads coordinates and weights, builds the histogram plan (autotuned when
// asked), runs the pipeline once (which fixes the count digits of the transform) and leaves the
// result in d_I / d_hist.
int batch_build(xns_batch *b, uint32_t nstruct, const uint32_t *nel, const uint32_t *n_el, const double *xyz,
                uint32_t nhist, double bin, const double *q, uint32_t nq, int source, const double *const *ff,
                const double *sl, int polar, double lambda, int autotune) {
  xns_ctx *ctx = b->ctx;
  if (!nel || !n_el || !xyz || !q || nstruct == 0 || nq == 0 || nhist == 0 || !(bin > 0))
    return xns_fail(ctx, XNS_ERR_ARG, "batch: null pointer or zero size");
  // the transform's grid has one row of CTAs per structure
  if (nstruct > 65535) return xns_fail(ctx, XNS_ERR_ARG, "batch: at most 65535 structures per batch");
  b->nstruct = nstruct;
  b->nq = nq;
  b->nhist = nhist;
  b->polar = polar;
  b->lambda = lambda;
  // elements and structures
  std::vector<const double *> table;
  std::vector<StructInfo> si(nstruct);
  uint32_t g = 0, cls = 0;
  size_t atoms = 0;
  for (uint32_t s = 0; s < nstruct; s++) {
    if (nel[s] == 0) return xns_fail(ctx, XNS_ERR_ARG, "batch: a structure without elements");
    si[s].cls_base = cls;
    si[s].e0 = g;
    si[s].nel = nel[s];
    si[s].ntot = 0;
    for (uint32_t e = 0; e < nel[s]; e++, g++) {
      table.push_back(xyz + 3 * atoms);
      atoms += n_el[g];
      si[s].ntot += n_el[g];
    }
    cls += xns_npairs(nel[s]);
  }
  if (atoms >= (1ull << 32)) return xns_fail(ctx, XNS_ERR_ARG, "batch: more than 2^32 atoms");
  b->classes = cls;
  const uint32_t G = g;
  int st;
  DevCoords dc;
  if ((st = xns_upload_coords(ctx, table.data(), n_el, G, &dc))) return st;
  if ((st = xns_upload_weights(ctx, G, nq, source, ff, sl, &b->d_w))) return st;
  // tables: q, atoms per element, structure info
  const size_t tbytes = sizeof(double) * nq + sizeof(uint32_t) * G + sizeof(StructInfo) * nstruct + 64;
  void *vt, *vh;
  if ((st = xns_scratch(ctx, SLOT_BATCH, tbytes, &vt))) return st;
  if ((st = xns_pinned(ctx, tbytes, &vh))) return st;
  b->d_q = (double *)vt;
  b->d_si = (StructInfo *)(b->d_q + nq);
  b->d_nel = (uint32_t *)(b->d_si + nstruct);
  char *h = (char *)vh;
  memcpy(h, q, sizeof(double) * nq);
  memcpy(h + sizeof(double) * nq, si.data(), sizeof(StructInfo) * nstruct);
  memcpy(h + sizeof(double) * nq + sizeof(StructInfo) * nstruct, n_el, sizeof(uint32_t) * G);
  XNS_CUDA(ctx, cudaMemcpyAsync(vt, vh, tbytes - 64, cudaMemcpyHostToDevice, ctx->stream));
  void *vhist, *vG, *vI;
  if ((st = xns_scratch(ctx, SLOT_BATCH_HIST, sizeof(unsigned long long) * (size_t)cls * nhist, &vhist))) return st;
  if ((st = xns_scratch(ctx, SLOT_TC_OUT, sizeof(double) * (size_t)cls * nq, &vG))) return st;
  if ((st = xns_scratch(ctx, SLOT_OUT, sizeof(double) * (size_t)nstruct * nq, &vI))) return st;
  b->d_hist = (unsigned long long *)vhist;
  b->d_G = (double *)vG;
  b->d_I = (double *)vI;

  HistSet hs;
  hs.x = dc.x;
  hs.y = dc.y;
  hs.z = dc.z;
  hs.el_off = dc.off_el;
  hs.el_n = dc.n_el;
  for (uint32_t s = 0; s < nstruct; s++) hs.st.push_back({si[s].e0, si[s].nel});

  if (autotune) {  // time the histogram launch for each candidate plan; keep the fastest
    static const HistTuning cand[] = {{56, HIST_WIN_MAX}, {32, HIST_WIN_MAX}, {96, HIST_WIN_MAX}, {56, 16 * 1024}};
    double best = 1e300;
    for (const HistTuning &t : cand) {
      HistLaunch L;
      if ((st = xns_hist_plan(ctx, hs, nhist, bin, b->d_hist, t, &L))) return st;
      if ((st = xns_stage_begin(ctx, STAGE_HIST))) return st;
      if ((st = xns_hist_enqueue(ctx, L))) return st;
      if ((st = xns_stage_end(ctx, STAGE_HIST))) return st;
      if ((st = xns_hist_check(ctx, L))) return st;
      const double ms = xns_last_stage_ms(ctx, STAGE_HIST);
      if (ms >= 0 && ms < best) {
        best = ms;
        b->tune = t;
      }
    }
    b->tuned_ms = best;
  }
  if ((st = xns_hist_plan(ctx, hs, nhist, bin, b->d_hist, b->tune, &b->hl))) return st;
  if ((st = xns_stage_begin(ctx, STAGE_HIST))) return st;
  if ((st = xns_hist_enqueue(ctx, b->hl))) return st;
  if ((st = xns_stage_end(ctx, STAGE_HIST))) return st;
  if ((st = xns_hist_check(ctx, b->hl))) return st;
  unsigned long long maxc = 0;
  if ((st = xns_tc_max_count(ctx, b->d_hist, cls, nhist, nhist, &maxc))) return st;
  if ((st = xns_tc_exact_plan(ctx, b->d_hist, cls, nhist, nhist, bin, q, nq, maxc, b->d_G, &b->xl, true))) return st;
  if ((st = xns_stage_begin(ctx, STAGE_IQ))) return st;
  if ((st = xns_tc_exact_enqueue(ctx, b->xl))) return st;
  if ((st = batch_epilogue(b))) return st;
  if ((st = xns_stage_end(ctx, STAGE_IQ))) return st;
  return xns_tc_exact_check(ctx, b->xl);
}

int batch_copy_out(xns_batch *b, double *I, uint64_t *hist) {
  xns_ctx *ctx = b->ctx;
  if (I) XNS_CUDA(ctx, cudaMemcpyAsync(I, b->d_I, sizeof(double) * (size_t)b->nstruct * b->nq, cudaMemcpyDeviceToHost,
                                       ctx->stream));
  if (hist)
    XNS_CUDA(ctx, cudaMemcpyAsync(hist, b->d_hist, sizeof(uint64_t) * (size_t)b->classes * b->nhist,
                                  cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XNS_OK;
}

void batch_free(xns_batch *b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->ctx) xns_destroy(b->ctx);
  delete b;
}

int batch_new(xns_ctx *parent, xns_batch **out) {
  *out = nullptr;
  xns_batch *b = new xns_batch();
  const int st = xns_create(parent->device, &b->ctx);
  if (st) {
    parent->err = "batch: " + std::string(xns_last_error(b->ctx));
    batch_free(b);
    return st;
  }
  *out = b;
  return XNS_OK;
}

}  // namespace

void xns_batch_release_cache(xns_ctx *ctx) {
  if (ctx && ctx->batch_cache) {
    batch_free(ctx->batch_cache);
    ctx->batch_cache = nullptr;
  }
}

extern "C" {

int xns_batch_create(xns_ctx *ctx, uint32_t nstruct, const uint32_t *nel, const uint32_t *n_el, const double *xyz,
                     uint32_t nhist, double bin, const double *q, uint32_t nq, int source, const double *const *ff,
                     const double *sl, int polar, double lambda, int autotune, xns_batch **out) {
  if (!ctx || !out) return XNS_ERR_ARG;
  xns_batch *b;
  int st;
  if ((st = batch_new(ctx, &b))) return st;
  st = batch_build(b, nstruct, nel, n_el, xyz, nhist, bin, q, nq, source, ff, sl, polar, lambda, autotune);
  if (!st) {  // capture the replayable part
    cudaStreamBeginCapture(b->ctx->stream, cudaStreamCaptureModeThreadLocal);
    const int est = batch_enqueue(b);
    const cudaError_t ce = cudaStreamEndCapture(b->ctx->stream, &b->graph);
    if (est) st = est;
    else if (ce != cudaSuccess) st = xns_cuda_fail(b->ctx, ce, "cudaStreamEndCapture");
    else if (cudaGraphInstantiate(&b->exec, b->graph, 0) != cudaSuccess)
      st = xns_fail(b->ctx, XNS_ERR_CUDA, "batch: graph instantiation failed");
  }
  if (st) {
    ctx->err = b->ctx->err;
    batch_free(b);
    return st;
  }
  *out = b;
  return XNS_OK;
}

int xns_batch_run(xns_batch *b, double *I, uint64_t *hist) {
  if (!b) return XNS_ERR_ARG;
  int st;
  if ((st = xns_timer_start(b->ctx))) return st;
  XNS_CUDA(b->ctx, cudaGraphLaunch(b->exec, b->ctx->stream));
  b->ctx->launches++;
  if ((st = xns_timer_stop(b->ctx))) return st;
  if ((st = batch_check(b))) return st;
  return batch_copy_out(b, I, hist);
}

double xns_batch_last_ms(const xns_batch *b) { return b ? xns_last_kernel_ms(b->ctx) : -1.0; }

const char *xns_batch_last_error(const xns_batch *b) { return b ? xns_last_error(b->ctx) : "null batch"; }

double xns_batch_tuning(const xns_batch *b, uint32_t *cell_target, uint32_t *window_bins) {
  if (!b) return -1.0;
  if (cell_target) *cell_target = b->tune.cell_target;
  if (window_bins) *window_bins = b->tune.win;
  return b->tuned_ms;
}

void xns_batch_destroy(xns_batch *b) { batch_free(b); }

int xns_calc_batch_debye_hist(xns_ctx *ctx, uint32_t nstruct, const uint32_t *nel, const uint32_t *n_el,
                              const double *xyz, uint32_t nhist, double bin, const double *q, uint32_t nq, int source,
                              const double *const *ff, const double *sl, int polar, double lambda, double *I,
                              uint64_t *hist) {
  if (!ctx) return XNS_ERR_ARG;
  if (!I) return xns_fail(ctx, XNS_ERR_ARG, "batch: null output");
  int st;
  // one-shot calls share a private batch kept by the context: its working memory and the transform's
  // sinc planes persist between calls with the same q mesh and bin grid
  if (!ctx->batch_cache && (st = batch_new(ctx, &ctx->batch_cache))) return st;
  xns_batch *b = ctx->batch_cache;
  const uint64_t l0 = b->ctx->launches;
  if ((st = xns_timer_start(b->ctx)) == 0)
    st = batch_build(b, nstruct, nel, n_el, xyz, nhist, bin, q, nq, source, ff, sl, polar, lambda, 0);
  if (!st) st = xns_timer_stop(b->ctx);
  if (!st) st = batch_copy_out(b, I, hist);
  if (st) {
    ctx->err = b->ctx->err;
    batch_free(b);  // a failed call may leave the private context in any state: start afresh next time
    ctx->batch_cache = nullptr;
  } else {
    ctx->last_ms = b->ctx->last_ms;
    ctx->launches += b->ctx->launches - l0;
  }
  return st;
}

}  // extern "C"
