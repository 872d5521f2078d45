// Internal definitions shared by the xns_b200 CUDA sources.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "xns_b200.h"

#define XNS_PI 3.1415926535897932384626433832795028841971693993  // typedefs.h:73
#define XNS_MAX_DEVICES 64  // devices tracked by the once-per-device kernel attribute settings

// Scratch slots: each is a grow-only device buffer owned by the context.
enum ScratchSlot {
  SLOT_COORDS_AOS = 0,  // staging for the caller's packed x y z triples
  SLOT_COORDS_SOA,      // x[], y[], z[] (FP64), element-major
  SLOT_HIST,            // u64 histogram
  SLOT_SEGPAIRS,        // tile-pair schedule
  SLOT_PARTIAL,         // per-CTA FP64 partial sums
  SLOT_WEIGHTS,         // per-element weights on the q mesh
  SLOT_QMESH,           // q values (FP64)
  SLOT_OUT,             // device copy of an output
  SLOT_OUT2,
  SLOT_FLAGS,           // error counters
  SLOT_AUX,
  SLOT_HSORT,           // histogram plan: cell-sorted coordinates and per-atom cell ids
  SLOT_HCELL,           // histogram plan: per-cell counts, offsets, cursors
  SLOT_HTILE,           // histogram plan: tiles (atom ranges with bounding boxes)
  SLOT_HLIST,           // histogram plan: tile pairs sorted by (element pair, distance bucket)
  SLOT_HTMP,            // histogram plan: tile pairs and keys in enumeration order (before the sort)
  SLOT_HKEY,            // histogram plan: bucket counts / offsets and small tables
  SLOT_TC_A,            // split-BF16 sinc matrix (hi and lo planes, tensor-core tile order)
  SLOT_TC_B,            // split-BF16 histogram columns (hi and lo planes)
  SLOT_TC_OUT,          // FP64 sinc-transform output (columns x q)
  SLOT_X_A,             // integer-digit planes: the sinc matrix (a q mesh used again) or the 2D plane's A
  SLOT_X_Q,             // the exact transform's q mesh
  SLOT_HFLAGS,          // histogram: out-of-range count and run queue
  SLOT_BATCH,           // batched ensemble: coordinates, schedules and per-structure tables
  SLOT_BATCH_HIST,      // batched ensemble: histograms
  SLOT_ATOMS,           // structure builder: the last build's atoms (x y z doubles, element-major)
  SLOT_EPS_HIST,        // sinc engine: the +1e-8 distance histogram
  SLOT_EPS_T,           // sinc engine: the +1e-8 sums per class and q
  SLOT_SPLIT,           // angle-split transform: cos / sin tables, weighted histogram columns, partial sums
  SLOT_COUNT
};

struct xns_ctx {
  int device = 0;
  int num_sms = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // kernel-only events of the last call: stage k (0 histogram, 1 PDF, 2 I(q) transform, 3 Debye
  // sum, 4 2D amplitude, 5 structure builder's site merge, 6 its atom-writing pass) ran between
  // ev_stage[2k] and ev_stage[2k+1]
  static const int NSTAGE = 7;
  cudaEvent_t ev_stage[2 * NSTAGE] = {};
  unsigned stage_mask = 0;
  double last_ms = 0;
  uint64_t launches = 0;
  std::string err;
  void *slot_ptr[SLOT_COUNT] = {};
  size_t slot_size[SLOT_COUNT] = {};
  size_t mem_limit = 0;  // cap on the sum of slot_size (0: none), xns_set_memory_limit
  unsigned long long inject_stall_ns = 0;  // xns_inject_pipeline_stall: consumed by the next digit GEMM
  bool debye_tc = true;                    // xns_debye_tensor_cores: the Debye sum on the integer tensor cores
  void *pinned = nullptr;  // pinned host staging
  size_t pinned_size = 0;
  // the sinc matrix held in SLOT_TC_A was built for this q mesh, bin width and K extent
  std::vector<double> tc_q;
  double tc_bin = 0;
  uint32_t tc_kt = 0;
  // the integer-digit sinc planes in SLOT_X_A were made for this q mesh, bin width and K extent; the
  // last mesh the exact transform saw (a second use builds the planes)
  std::vector<double> x_q, x_seen_q;
  double x_bin = 0, x_seen_bin = 0;
  uint32_t x_kt = 0, x_seen_kt = 0;
  // private batch reused by the one-shot batched entry point (batch.cu)
  struct xns_batch *batch_cache = nullptr;
  // atoms per element of the last structure build (SLOT_ATOMS)
  std::vector<uint32_t> atoms_n;
};
void xns_batch_release_cache(xns_ctx *ctx);

// One entry of the tile-pair schedule: atoms [a0, a0+na) against [b0, b0+nb) of the SoA arrays.
// same != 0: the two ranges are the same segment and only pairs i < j count (CalcFunctions.cpp:576).
struct SegPair {
  uint32_t a0, na, b0, nb;
  uint32_t cls;    // output class (element pair t for histograms; accumulator row for Debye)
  uint32_t same;
  uint32_t ta, tb; // tiles along a and b
  uint32_t ratio;  // a-tiles per b-tile (tile_b / tile_a)
  uint32_t pad;
  unsigned long long tile_begin;  // prefix over the schedule
};

// Status helpers (return an int status and record the message in the context).
int xns_fail(xns_ctx *ctx, int status, const std::string &msg);
int xns_cuda_fail(xns_ctx *ctx, cudaError_t e, const char *what);
#define XNS_CUDA(ctx, call)                                   \
  do {                                                        \
    cudaError_t _e = (call);                                  \
    if (_e != cudaSuccess) return xns_cuda_fail(ctx, _e, #call); \
  } while (0)
#define XNS_LAUNCHED(ctx)                                            \
  do {                                                               \
    (ctx)->launches++;                                               \
    cudaError_t _e = cudaGetLastError();                             \
    if (_e != cudaSuccess) return xns_cuda_fail(ctx, _e, "kernel launch"); \
  } while (0)

// Grow-only device scratch.
int xns_scratch(xns_ctx *ctx, ScratchSlot slot, size_t bytes, void **out);
// Pinned host staging (grow-only).
int xns_pinned(xns_ctx *ctx, size_t bytes, void **out);

// Device-resident coordinates in SoA FP64 form, element-major.
struct DevCoords {
  const double *x, *y, *z;
  uint32_t ntot;
  std::vector<uint32_t> n_el;
  std::vector<uint32_t> off_el;
};
// Copies per-element packed x y z triples to the device as SoA (one async copy per element + a
// transpose kernel).
int xns_upload_coords(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel, DevCoords *dc);

// Histogram on device coordinates; d_hist receives P*nhist counts.  Used by the host-buffer entry
// points and by the fused pipelines.
int xns_hist_device(xns_ctx *ctx, const DevCoords &dc, uint32_t nhist, double bin, unsigned long long *d_hist);
// Histogram -> I(q) on a device histogram.  d_w: per-element weights on the q mesh (nel x nq, FP64).
int xns_hist_iq_device(xns_ctx *ctx, const unsigned long long *d_hist, const uint32_t *n_el, uint32_t nel, uint32_t nhist,
                       double bin, const double *q, uint32_t nq, const double *d_w, int polar, double lambda, double *d_I);
// PDF on a device histogram; d_pdf receives (1+P)*nhist doubles.
int xns_pdf_device(xns_ctx *ctx, const unsigned long long *d_hist, const uint32_t *n_el, uint32_t nel, uint32_t nhist,
                   double bin, int pdftype, double p0, const double *sl, double *d_pdf);
// Per-element weights on the q mesh as a device array (nel x nq): ff rows (X-ray) or sl (neutron).
int xns_upload_weights(xns_ctx *ctx, uint32_t nel, uint32_t nq, int source, const double *const *ff, const double *sl,
                       double **d_w);

// Uniform mesh test: returns true when q[i] == q[0] + i*dq bit for bit with dq = (q[n-1]-q[0])/(n-1)
// rounded as the reference builds it, and reports q0 and dq.
bool xns_uniform_mesh(const double *q, uint32_t nq, double *q0, double *dq);

// Event timing around a sequence of kernels on ctx->stream.
int xns_timer_start(xns_ctx *ctx);
int xns_timer_stop(xns_ctx *ctx);
// Kernel-only stage timing (see xns_ctx::ev_stage).
enum { STAGE_HIST = 0, STAGE_PDF = 1, STAGE_IQ = 2, STAGE_DEBYE = 3, STAGE_2D = 4, STAGE_MERGE = 5, STAGE_FILL = 6 };
int xns_stage_begin(xns_ctx *ctx, int k);
int xns_stage_end(xns_ctx *ctx, int k);

static inline uint32_t xns_npairs(uint32_t nel) { return nel * (nel + 1) / 2; }
// Device-resident x y z triples (element-major) -> SoA scratch (no host copy).
int xns_coords_from_device(xns_ctx *ctx, const double *xyz_dev, const uint32_t *n_el, uint32_t nel, DevCoords *dc);
