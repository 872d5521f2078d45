/* xns_b200 -- B200 (sm_100a) implementation of the XaNSoNS scattering calc functions.
 *
 * C ABI: plain pointers and sizes, int status, caller-owned outputs.  The library owns its device
 * memory and its CUDA stream; every call is synchronous with respect to the host buffers it is given.
 *
 * Conventions shared by all entry points
 *   - Coordinates are passed per element, exactly as the reference's vector<vect3d<double>> ra[Nel]
 *     holds them: xyz_el[e] points at n_el[e] packed x y z double triples (vect3d<double> is three
 *     doubles, typedefs.h:83-142, so &ra[e][0].x can be passed directly).
 *   - Element pairs (a <= b) are numbered in the reference's loop order (a outer, b inner);
 *     P = nel(nel+1)/2.  Histograms are element-pair major: hist[t*nhist + k].
 *   - source: XNS_NEUTRON uses sl[e] (scattering lengths); XNS_XRAY uses ff[e][iq] (form factor on the
 *     q mesh), as the reference's SL / FF vectors (ReadXML.cpp:329-331).
 *   - The q mesh is the array the reference builds, q[i] = qmin + i*(qmax-qmin)/N (ReadXML.cpp:220-222);
 *     uniform meshes take the fast path, any other mesh a per-term kernel.
 *   - Errors: a non-zero status; xns_last_error() gives a one-line description.  On error the
 *     outputs are unspecified.  No entry point falls back to CPU computation.
 */
#ifndef XNS_B200_H
#define XNS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define XNS_OK 0
#define XNS_ERR_ARG 1      /* invalid argument */
#define XNS_ERR_CUDA 2     /* CUDA runtime error (message in xns_last_error) */
#define XNS_ERR_NODEV 3    /* no sm_100 device / library not built for it */
#define XNS_ERR_RANGE 4    /* a pair distance fell beyond the histogram (reference: out-of-bounds write) */
#define XNS_ERR_NOMEM 5    /* device allocation failed */
#define XNS_ERR_LIMIT 6    /* a size beyond the fixed limits of xns_int_1d_hist_noalloc */

/* typedefs.h:50-56 */
#define XNS_NEUTRON 0
#define XNS_XRAY 1
#define XNS_RDF 0
#define XNS_PDF 1
#define XNS_RPDF 2
/* scenarios, typedefs.h:43-47 */
#define XNS_DEBYE_HIST 2
#define XNS_PDF_ONLY 3
#define XNS_DEBYE_PDF 4

typedef struct xns_ctx xns_ctx;

/* Context on one CUDA device (device = -1 picks the current one).  Replaces the reference's
 * SetDeviceCuda (CalcFunctionsCUDA.cu:1485-1519): it requires compute capability 10.x. */
int xns_create(int device, xns_ctx **out);
void xns_destroy(xns_ctx *ctx);
const char *xns_last_error(const xns_ctx *ctx);
const char *xns_status_string(int status);
/* Run on the caller's stream (a cudaStream_t) instead of the library's own; NULL restores it. */
int xns_set_stream(xns_ctx *ctx, void *stream);
/* Caps the device scratch the calc functions keep in the context between calls (their grow-only
 * buffers) at bytes; 0 removes the cap.  A call that would need more returns XNS_ERR_NOMEM before
 * queueing any work, and the context stays usable.  If the context already holds more than the new
 * cap, that scratch is released first (the context's stream is synchronised).  For a service with a
 * fixed device-memory budget per context; no counterpart in the reference. */
int xns_set_memory_limit(xns_ctx *ctx, uint64_t bytes);
/* Failure-path test of the tensor-core pipelines: the next tensor-core transform on this context
 * (xns_hist_transform_exact, the batched ensembles' transform or the 2D plane; not the calc functions'
 * FP64 histogram transform) runs with its copy warp issuing no copies
 * and every pipeline wait bounded by wait_limit_ns (at most 2 s, the kernels' own bound).  Its waits
 * run out, the kernel releases its tensor memory and returns, and that call fails with XNS_ERR_CUDA
 * ("a pipeline wait ran out of time"); the context stays usable and the following calls run
 * normally.  Affects one call.  No counterpart in the reference. */
int xns_inject_pipeline_stall(xns_ctx *ctx, uint64_t wait_limit_ns);
/* Path of the exact Debye double sum (xns_calc_int_debye, xns_calc_int_partial_debye and their
 * shards) on a uniform q mesh: on (the default), the integer tensor cores (terms as 8-bit digit products
 * summed exactly in tensor memory, then in FP64) whenever the largest pair distance is at most 256
 * times the smallest nonzero one; off, or outside that range or on a mesh that is not uniform, the
 * FP32 sine recurrence on the FMA pipe.  Both agree with the reference within its tolerance; the
 * tensor-core path is the more accurate and the faster.  No counterpart in the reference. */
int xns_debye_tensor_cores(xns_ctx *ctx, int on);
/* Device time of the most recent call's kernels, in milliseconds (CUDA events). */
double xns_last_kernel_ms(const xns_ctx *ctx);
/* Number of kernels the library launched since the context was created. */
uint64_t xns_kernel_launches(const xns_ctx *ctx);
/* Kernel-only device time (CUDA events on the library's stream) of one stage of the most recent call:
 * 0 histogram, 1 PDF, 2 histogram -> I(q), 3 Debye double sum, 4 2D amplitude, 5 the structure
 * builder's site merge, 6 its atom-writing pass (the last block's); -1 if it did not run. */
double xns_last_stage_ms(const xns_ctx *ctx, int stage);

/* ---- host-buffer entry points (what the reference's calc functions become) ---------------------- */

/* Pair-distance histogram.  Replaces calcHist (CalcFunctions.cpp:757-809) and calcHistCuda
 * (CalcFunctionsCUDA.cu:855-920).  hist: P*nhist counts, bit-identical to the reference's FP64
 * (unsigned int)(|ri-rj|/bin).  XNS_ERR_RANGE if some distance maps to a bin >= nhist.  Structures of
 * any size: beyond 2^28 tile pairs (about 2e6 atoms) the count runs in passes (xns_calc_hist_passes). */
int xns_calc_hist(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel, uint32_t nhist, double bin,
                  uint64_t *hist);

/* xns_calc_hist in passes: the tile pairs of the spatial plan are enumerated and taken at most
 * max_tile_pairs at a time (16 bytes of device memory each; 0 = 2^28, the default of every histogram
 * entry point), each pass adding into one histogram, so that structures of any size fit the device;
 * the result equals xns_calc_hist's. */
int xns_calc_hist_passes(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel, uint32_t nhist,
                         double bin, uint64_t max_tile_pairs, uint64_t *hist);

/* Histogram -> I(q).  Replaces calcInt1DHist (CalcFunctions.cpp:810-911) and calcInt1DHistCuda
 * (CalcFunctionsCUDA.cu:988-1045).  ff: nel pointers to nq doubles (X-ray) or NULL; sl: nel doubles
 * (neutron) or NULL.  I: nq doubles, already divided by ntot and polarisation-corrected if polar. */
int xns_calc_int_1d_hist(xns_ctx *ctx, const uint64_t *hist, const uint32_t *n_el, uint32_t nel, uint32_t nhist, double bin,
                         const double *q, uint32_t nq, int source, const double *const *ff, const double *sl, int polar,
                         double lambda, double *I);

/* PDF / RDF / rPDF from a histogram.  Replaces the PDF branch of calcPDFandDebye
 * (CalcFunctions.cpp:919-960) and calcPDFCuda (CalcFunctionsCUDA.cu:1048-1160).  sl: the per-element
 * weights the reference uses there.  pdf: (1+P)*nhist doubles, total first. */
int xns_calc_pdf(xns_ctx *ctx, const uint64_t *hist, const uint32_t *n_el, uint32_t nel, uint32_t nhist, double bin,
                 int pdftype, double p0, const double *sl, double *pdf);

/* Histogram + PDF + I(q) in one device pass.  Replaces calcPDFandDebye (CalcFunctions.cpp:912-968) and
 * calcPDFandDebyeCuda (CalcFunctionsCUDA.cu:1078-1160).  scenario: XNS_DEBYE_HIST, XNS_PDF_ONLY or
 * XNS_DEBYE_PDF; I (nq) is written for DEBYE_HIST / DEBYE_PDF, pdf ((1+P)*nhist) for PDF_ONLY / DEBYE_PDF.
 * hist_out, when non-NULL, receives the P*nhist counts as well. */
int xns_calc_pdf_and_debye(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel, uint32_t nhist,
                           double bin, int scenario, int pdftype, double p0, const double *q, uint32_t nq, int source,
                           const double *const *ff, const double *sl, int polar, double lambda, double *I, double *pdf,
                           uint64_t *hist_out);

/* Exact Debye double sum.  Replaces calcIntDebye (CalcFunctions.cpp:547-633) and calcIntDebyeCuda
 * (CalcFunctionsCUDA.cu:1276-1355).  I: nq doubles. */
int xns_calc_int_debye(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel, const double *q,
                       uint32_t nq, int source, const double *const *ff, const double *sl, int polar, double lambda, double *I);

/* Debye double sum split into block-pair parts.  Replaces calcIntPartialDebye (CalcFunctions.cpp:634-756)
 * and calcIntPartialDebyeCuda (CalcFunctionsCUDA.cu:1377-1481).  n_el_block[e*nblocks+b] = atoms of
 * element e in block b (ra[e] holds block 0's atoms first).  I: (1 + nblocks(nblocks+1)/2)*nq, total first. */
int xns_calc_int_partial_debye(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel,
                               uint32_t nblocks, const uint32_t *n_el_block, const double *q, uint32_t nq, int source,
                               const double *const *ff, const double *sl, int polar, double lambda, double *I);

/* 2D pattern on the reference's polar (q, phi) mesh, averaged over the Euler-angle mesh.  Replaces
 * calcInt2D (CalcFunctions.cpp:969-1091) and calcInt2DCuda (CalcFunctionsCUDA.cu:653-776).  Euler angles
 * in radians; convention as typedefs.h:59-70.  I2D: nq x nfi row-major; I: nq (phi average). */
int xns_calc_int_2d(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel, const double *q,
                    uint32_t nq, uint32_t nfi, const double *euler_min, const double *euler_max, const uint32_t *euler_n,
                    uint32_t convention, double lambda, int source, const double *const *ff, const double *sl, int polar,
                    double *I2D, double *I);

/* The rotation matrix of calcRotMatrix (CalcFunctions.cpp:46-115) for Euler angles euler[0..2] (radians)
 * in convention 0..11 (typedefs.h:59-70), row-major, as xns_calc_int_2d applies it per orientation.
 * Host-only; needs no device.  Use it to orient coordinates for xns_calc_amp_plane. */
void xns_rot_matrix(const double euler[3], uint32_t convention, double m[9]);

/* ---- device-buffer entry points ----------------------------------------------------------------- */

/* calcPDFandDebye (CalcFunctions.cpp:912-968) on device-resident data: xyz_dev is a device array of
 * sum(n_el) x y z double triples, element-major (the reference's dataCopyCUDA staging,
 * CalcFunctionsCUDA.cu:1522-1555, kept in FP64); hist_dev (P*nhist), I_dev (nq) and pdf_dev
 * ((1+P)*nhist) are device arrays.  q, ff, sl stay host arrays.  Synchronous: returns after the
 * kernels finished; xns_last_kernel_ms() gives their device time. */
int xns_pdf_and_debye_device(xns_ctx *ctx, const double *xyz_dev, const uint32_t *n_el, uint32_t nel, uint32_t nhist,
                             double bin, int scenario, int pdftype, double p0, const double *q, uint32_t nq, int source,
                             const double *const *ff, const double *sl, int polar, double lambda, double *I_dev,
                             double *pdf_dev, uint64_t *hist_dev);

/* ---- one structure over several GPUs ---------------------------------------------------------------- */

/* One shard of calcHist (CalcFunctions.cpp:757-809): the counts of this shard's share of the atom
 * pairs.  The plan (spatial sort, tile pairs, runs) is the whole structure's; shard s of nshard keeps
 * every nshard-th run of its size-sorted run list and every nshard-th of the tile pairs too wide for a
 * window, so the shares balance and the histograms of shards 0..nshard-1 add up, bin by bin, to
 * xns_calc_hist's exactly.  Each GPU (rank) computes its shard; a sum across ranks (an NCCL all-reduce
 * of P*nhist u64, the reference's MPI_Reduce of rij_hist, CalcFunctions.cpp:804-807) gives the
 * histogram, from which I(q) and the PDF follow on any rank.  Host-buffer and device-buffer forms. */
int xns_calc_hist_shard(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel, uint32_t nhist,
                        double bin, uint32_t shard, uint32_t nshard, uint64_t *hist);
int xns_hist_shard_device(xns_ctx *ctx, const double *xyz_dev, const uint32_t *n_el, uint32_t nel, uint32_t nhist,
                          double bin, uint32_t shard, uint32_t nshard, uint64_t *hist_dev);
/* One shard of calcIntDebye / calcIntPartialDebye (CalcFunctions.cpp:547-756): the intensity of the
 * tile pairs w with w % nshard == shard, the self term (sum of N_e w_e^2) on shard 0 only, normalised
 * and polarised as the whole.  The outputs of shards 0..nshard-1 add up to xns_calc_int_debye's /
 * xns_calc_int_partial_debye's (up to FP64 summation order): an all-reduce of nq (or (1 + parts) nq)
 * doubles across ranks, the reference's MPI_Reduce of Itemp (CalcFunctions.cpp:613, :729).
 * n_el_block: as xns_calc_int_partial_debye, or NULL with nblocks = 1. */
int xns_calc_int_debye_shard(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel, uint32_t nblocks,
                             const uint32_t *n_el_block, const double *q, uint32_t nq, int source, const double *const *ff,
                             const double *sl, int polar, double lambda, uint32_t shard, uint32_t nshard, double *I);
/* The rest of calcPDFandDebye (CalcFunctions.cpp:912-968) on a device histogram, e.g. the sum of the
 * shards: PDF (pdf_dev, (1+P)*nhist) and / or I(q) (I_dev, nq) as xns_pdf_and_debye_device gives them. */
int xns_pdf_and_debye_from_hist_device(xns_ctx *ctx, const uint64_t *hist_dev, const uint32_t *n_el, uint32_t nel,
                                       uint32_t nhist, double bin, int scenario, int pdftype, double p0, const double *q,
                                       uint32_t nq, int source, const double *const *ff, const double *sl, int polar,
                                       double lambda, double *I_dev, double *pdf_dev);

/* ---- allocation-free entry point ------------------------------------------------------------------ */

/* Histogram -> I(q) that allocates no device memory.  No counterpart in the reference: it serves
 * callers that cannot call cudaMalloc -- a plugin whose host framework owns all device memory and
 * hands it buffers, or a service whose memory budget is fixed at start-up.  The caller passes the
 * histogram (hist_dev: P*nhist u64) and the output (I_dev: nq doubles) as device buffers it owns.
 * Intermediates live in one file-scope device array of XNS_NOALLOC_SCRATCH_BYTES that every GPU
 * loading the library holds until exit.
 * Accuracy: the result is xns_calc_int_1d_hist's quantity computed another way -- an FP32 sine
 * recurrence over the bins with FP64 seeds and FP64 sums (the engine of the exact Debye sum) instead
 * of the FP64 angle-split sums -- and agrees with it within 1e-5 relative at every q, the deep
 * low-q minima of I(q) included (the GPU tests check a 10-cell rock-salt cube at 0.001 A on 4096 q).
 * Limits: at most XNS_NOALLOC_MAX_ELEMENTS elements; at most XNS_NOALLOC_MAX_Q q points on a uniform
 * mesh and XNS_NOALLOC_MAX_Q_NONUNIFORM on any other; and the array must hold, each region rounded up
 * to 256 bytes, the weights and the q mesh ((nel + 1) * nq * 8 bytes), the pair tables ((2P + nel) * 4),
 * the +1e-8 histogram (P * nb * 8, nb = min(4096, nhist * bin / 0.05 + 2)), its sums (P * nq * 8) and
 * at least one CTA's partial sums (P * nq * 8).  Larger sizes return XNS_ERR_LIMIT before any work is
 * queued.  Runs on the current device and the given stream (NULL = default stream); X-ray form factors
 * and a non-uniform q mesh are copied from the caller's host arrays with cudaMemcpyAsync, which waits
 * for the copy when that host memory is pageable.  The first call on a device looks up the array's
 * device address: make it before any stream capture.  Calls share the array: calls that overlap on the
 * GPU (other streams, other host threads) race on it. */
#define XNS_NOALLOC_SCRATCH_BYTES (16u << 20)
#define XNS_NOALLOC_MAX_ELEMENTS 16
#define XNS_NOALLOC_MAX_Q 8192
#define XNS_NOALLOC_MAX_Q_NONUNIFORM 2048
int xns_int_1d_hist_noalloc(const uint64_t *hist_dev, const uint32_t *n_el, uint32_t nel, uint32_t nhist, double bin,
                            const double *q, uint32_t nq, int source, const double *const *ff, const double *sl, int polar,
                            double lambda, double *I_dev, void *stream);

/* ---- split-precision tensor-core transform -------------------------------------------------------- */

/* The histogram -> I(q) contraction of calcInt1DHist (CalcFunctions.cpp:855-864) for ncols histogram
 * columns at once, on the tensor cores in split-BF16 (3 products, FP32 accumulation, FP64 cross-CTA
 * sums):  G[c*nq + i] = sum_k hist[c*nh + k] * sin(q_i r_k) / (q_i r_k),  r_k = (k + 0.5) * bin.
 * No weights, no self term and no 1/N: the column-level kernel the batched entry points build on.
 * Relative error of G against FP64 below 1e-4 (typically 1e-5).  The sinc matrix is cached in the
 * context for the last (q mesh, bin, nh / 64) and rebuilt when they change. */
int xns_hist_transform_bf16x3(xns_ctx *ctx, const uint64_t *hist, uint32_t ncols, uint32_t nh, double bin,
                              const double *q, uint32_t nq, double *G);

/* The same G with exact accumulation on the BF16 tensor cores: the sinc matrix (FP64, with the
 * reference's +1e-8 in the denominator) as five base-256 integer digits, the counts as two to four
 * base-256 digits, all digit products summed exactly (integers below 2^24 in the FP32 accumulator,
 * flushed to FP64 every 128 bins).  G carries the FP64 sinc's error plus < 1e-12 per matrix
 * element, so I(q) stays within 1e-5 of FP64 even at the deep minima of small particles, where the
 * FP32-accumulated bf16x3 form loses precision.  Counts below 2^32 (XNS_ERR_LIMIT beyond). */
int xns_hist_transform_exact(xns_ctx *ctx, const uint64_t *hist, uint32_t ncols, uint32_t nh, double bin,
                             const double *q, uint32_t nq, double *G);

/* The same G in FP64 by angle splitting, the form xns_calc_int_1d_hist and the fused entry points use:
 * each bin distance r_k = R_h + r_l (R_h a multiple of 64 bins), sin(q r_k) = sin(q R_h) cos(q r_l) +
 * cos(q R_h) sin(q r_l), so the bin sum is an FP64 product with K = 64 against per-q tables of 64
 * cosines and sines, and the +1e-8 of the denominator is kept to first order (sum_k n_k sin(q r_k) / r_k^2
 * by an FP64 rotation over the bins, per bin below 20 A and in 0.02 A bins beyond, within 5e-12 of the
 * terms; the next order is below 1e-14 of the terms).  No sinc matrix and no cache: every call costs
 * the same.  G carries FP64 rounding (about 1e-13 of its terms).  Scratch: 1 KB per q point, at most 32
 * bytes per bin, 8 bytes per column and bin below 20 A, and the partial sums (at most 32 bytes per q
 * point and split, about 16 x SMs x 64 / nq splits).  Counts below 2^53. */
int xns_hist_transform_split(xns_ctx *ctx, const uint64_t *hist, uint32_t ncols, uint32_t nh, double bin,
                             const double *q, uint32_t nq, double *G);

/* ---- 2D intensity on a flat Cartesian q plane ------------------------------------------------------ */

/* The calcInt2D amplitude (CalcFunctions.cpp:1026-1046) for the detector plane normal to the beam in the
 * limit of a flat Ewald surface: I[iy * nqx + ix] = |sum_e f_e(|q|) sum_{j in e} exp(i (qx x_j + qy y_j))|^2
 * / N with qx = qx0 + ix dqx, qy = qy0 + iy dqy; coordinates as given (pre-rotate them for another
 * orientation).  Since exp(i (qx x + qy y)) factorises, the sum is a complex matrix product over atoms,
 * run on the tensor cores with four base-256 integer digits per cos / sin value and exact accumulation
 * (measured error 2e-7 of the pattern's maximum).  X-ray: coef holds 9 numbers per element, f(q) = sum_k a_k exp(-b_k (q/4pi)^2) + c
 * as (a1..a4, b1..b4, c); neutron: sl.  No counterpart entry in the reference (its 2D mesh is polar on
 * the Ewald sphere: xns_calc_int_2d). */
int xns_calc_amp_plane(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel, double qx0,
                       double dqx, uint32_t nqx, double qy0, double dqy, uint32_t nqy, int source, const double *coef,
                       const double *sl, double *I);

/* ---- batched ensembles ------------------------------------------------------------------------------ */

/* No reference counterpart as one call: the reference evaluates one structure per run.  Per structure
 * the result is calcPDFandDebye's Debye_hist intensity (CalcFunctions.cpp:912-968): the histogram of
 * calcHist (:757-809, bit-exact) and the I(q) of calcInt1DHist (:810-911, exact transform, within 1e-5
 * of FP64).
 *
 * Inputs, for nstruct structures (1..65535):
 *   nel[s]      elements of structure s; G = sum nel elements in all;
 *   n_el[g]     atoms of element g (structure-major, then element order), g < G;
 *   xyz         all atoms as packed x y z doubles in that order (sum n_el triples);
 *   nhist, bin  one histogram grid for all structures (nhist >= every structure's need);
 *   sl[g] / ff[g][iq]  weights per element g (neutron / X-ray), as in the single-structure calls.
 * Outputs: I (nstruct x nq), hist (optional: classes x nhist u64, classes = sum P(nel[s]), structure s
 * owning its P(nel[s]) element pairs in the reference's order).
 *
 * xns_calc_batch_debye_hist does everything in one call.  xns_batch_create plans the ensemble (spatial
 * sort and tile pairs of all structures, optionally autotuned), runs it once and captures the launches
 * of the histogram, transform and epilogue in a CUDA graph; xns_batch_run replays that graph (for the
 * same coordinates, e.g. after changing nothing but wanting the result again, or for timing).  A batch
 * owns a private context (stream and working memory) on the caller's device. */
typedef struct xns_batch xns_batch;
int xns_calc_batch_debye_hist(xns_ctx *ctx, uint32_t nstruct, const uint32_t *nel, const uint32_t *n_el,
                              const double *xyz, uint32_t nhist, double bin, const double *q, uint32_t nq, int source,
                              const double *const *ff, const double *sl, int polar, double lambda, double *I,
                              uint64_t *hist);
int xns_batch_create(xns_ctx *ctx, uint32_t nstruct, const uint32_t *nel, const uint32_t *n_el, const double *xyz,
                     uint32_t nhist, double bin, const double *q, uint32_t nq, int source, const double *const *ff,
                     const double *sl, int polar, double lambda, int autotune, xns_batch **out);
int xns_batch_run(xns_batch *b, double *I, uint64_t *hist);
/* Device time of the last xns_batch_run (ms) and its error message. */
double xns_batch_last_ms(const xns_batch *b);
const char *xns_batch_last_error(const xns_batch *b);
/* The plan the autotuner kept (mean atoms per spatial cell, window bins) and its histogram time in ms
 * (-1 when the batch was created without autotuning). */
double xns_batch_tuning(const xns_batch *b, uint32_t *cell_target, uint32_t *window_bins);
void xns_batch_destroy(xns_batch *b);

/* ---- learned binning correction: a small MLP trained on the GPU ------------------------------------ */

/* No reference counterpart.  A 3-layer perceptron y = W3 gelu(W2 gelu(W1 x + b1) + b2) + b3 with FP32
 * master weights used in BF16 by hand-written forward and backward kernels (FP32 accumulation), trained
 * with Adam on a mean weighted squared error.  dims = {in, hidden, hidden, out}.  Parameters are laid
 * out W1 (hidden x in, row-major), b1, W2, b2, W3, b3.  x, t, y, grad are host buffers; w (per output
 * column loss weights) may be NULL.  The network owns a private context on the caller's device. */
typedef struct xns_mlp xns_mlp;
int xns_mlp_create(xns_ctx *ctx, const int *dims, uint64_t seed, xns_mlp **out);
void xns_mlp_destroy(xns_mlp *m);
const char *xns_mlp_last_error(const xns_mlp *m);
long xns_mlp_param_count(const xns_mlp *m);
int xns_mlp_get_params(xns_mlp *m, float *params);
int xns_mlp_set_params(xns_mlp *m, const float *params);
int xns_mlp_forward(xns_mlp *m, const float *x, int batch, float *y);
int xns_mlp_gradients(xns_mlp *m, const float *x, const float *t, const float *w, int batch, float *grad,
                      double *loss);
int xns_mlp_train(xns_mlp *m, const float *x, const float *t, const float *w, int n, int batch, int epochs, float lr,
                  double *loss);

/* Kernels of the learned correction.  h: a structure's weighted coarse histogram normalised by N s0
 * (so that I = s0 [1 + sum_k h_k sin(q r_k)/(q r_k)]), nh bins of width bin.
 * xns_binning_features: per bin the perceptron's XNS_BINNING_FEATURES inputs (log(1 + h) of the bin and
 * its 4 neighbours on each side, the neighbours' ratios to the bin, the bin position), X: nh x 18.
 * xns_binning_correction: dI(q) = s0 sum_k h_k [mu1_k D S'(q r_k) + m2_k D^2/2 S''(q r_k)], the second
 * order Taylor correction for within-bin offsets with moments mu = (mu1, m2) per bin (nh x 2, in units
 * of the bin width D); S = sin(q r)/(q r). */
#define XNS_BINNING_FEATURES 18
int xns_binning_features(xns_ctx *ctx, const double *h, uint32_t nh, float *X);
int xns_binning_correction(xns_ctx *ctx, const double *h, const float *mu, uint32_t nh, double bin, const double *q,
                           uint32_t nq, double s0, double *dI);

/* ---- structure builder ------------------------------------------------------------------------------ */

/* One block of the structure, as block::calcAtoms (CalcFunctions.cpp:251-392) reads it after the XML
 * reader prepared it (ReadXML.cpp:254-303: redefAtoms / redefSymm to Cartesian, centerAtoms, sortAtoms,
 * calcMean, calcRotMatrix of each copy).  Arrays are borrowed for the duration of the call. */
typedef struct xns_block {
  uint32_t natom;          /* sites of the asymmetric unit (block::Natom), element-sorted */
  uint32_t nid;            /* elements present in the block (block::Nid) */
  uint32_t nsymm;          /* symmetry operations (block::Nsymm, >= 1) */
  uint32_t ncopy;          /* copies (block::Ncopy, >= 1) */
  uint32_t ncell[3];       /* unit cells along e[0], e[1], e[2] (block::Ncell) */
  int32_t cutoff;          /* block::cutoff, radius rcut about r_mean */
  int32_t cutoff_copies;   /* block::cutoffcopies, radius rcut_copies about the mean copy position */
  int32_t ro_mol;          /* block::ro_mol: a random rotation per symmetry-equivalent molecule */
  const uint32_t *natom_el; /* [nid] sites of each element, in order (block::NatomEl) */
  const uint32_t *id;       /* [nid] global element index of each (block::id) */
  const double *r_atom;     /* [natom][3] site coordinates, Cartesian (block::rAtom) */
  const double *occ;        /* [natom] occupancies (block::occ) */
  const double *dev;        /* [natom] displacement widths (block::dev) */
  const double *p_symm;     /* [nsymm][3][3] rotation part, row k of operation s at [s][k] (block::pSymm[k][s]) */
  const double *r_symm;     /* [nsymm][3] translation part, Cartesian (block::rSymm) */
  const double *r_copy;     /* [ncopy][3] copy positions (block::rCopy) */
  const double *cf;         /* [ncopy][3][3] copy rotations, row k of copy c at [c][k] (block::cf[k][c]) */
  double e[3][3];           /* cell vectors (block::e) */
  double r_mean[3];         /* block::rMean */
  double rcut, rcut_copies, dev_mol;
} xns_block;

/* block::calcAtoms for each block in turn on the GPU.  The atoms of every block are appended, element
 * by element, in the reference's order (copy, cell x, y, z, site), and the result is kept in the
 * context as one device array of sum(n_el) x y z double triples, element-major (the xyz_dev layout of
 * xns_pdf_and_debye_device); *xyz_dev points at it until the next build or xns_destroy.
 *   n_el[nel]: atoms of each global element;  n_all (optional): atoms of each block element, blocks
 *   in order (block::NatomElAll, sum of nid entries).
 * Sites closer than 0.5 A (also across the +-2 neighbouring cells of every replicated axis) are merged
 * and filled by one random draw against their cumulative occupancy, as the reference does; the
 * random numbers come from Philox4x32-10 keyed by seed and indexed by (block, copy and cell, site,
 * purpose), so a build is reproducible for a seed (the reference seeds from the clock).
 * Sites per block below 2^31, atoms in all below 2^32 - 1, nel <= 64. */
int xns_build_atoms(xns_ctx *ctx, const xns_block *blocks, uint32_t nblocks, uint32_t nel, uint64_t seed,
                    uint32_t *n_el, uint32_t *n_all, const double **xyz_dev);
/* Copies the last build's atoms into host arrays: xyz_el[e] receives n_el[e] x y z triples. */
int xns_copy_atoms(xns_ctx *ctx, double *const *xyz_el);

/* ---- rearrangement correction ------------------------------------------------------------------------ */

/* One block as RearrangementInt (CalcFunctions.cpp:469-545) reads it: the block's sites (element-sorted,
 * Cartesian), per site the list of its neighbours read from the block's Rearrangement file
 * (block::readRearrangement, IO.cpp:198-230: positions, global element ids), Rcorr, and
 * coeff = Ncopy * Ncell.x * Ncell.y * Ncell.z * Nsymm as the reference forms it (unsigned int). */
typedef struct xns_rearr_block {
  uint32_t natom, nid;
  uint32_t rearrangement;     /* 0: the block contributes nothing (block::rearrangement) */
  uint32_t coeff;
  const uint32_t *natom_el;   /* [nid] sites per block element */
  const uint32_t *id;         /* [nid] global element index of each */
  const double *r_atom;       /* [natom][3] */
  const uint32_t *neighb_off; /* [natom + 1] CSR offsets into the neighbour arrays */
  const double *neighb_r;     /* [neighb_off[natom]][3] neighbour positions */
  const uint32_t *neighb_id;  /* [neighb_off[natom]] global element index of each neighbour */
  double rcorr;
} xns_rearr_block;

/* RearrangementInt (CalcFunctions.cpp:469-545) on the GPU: I0 (host, in / out; nq values, or
 * (1 + nblocks (nblocks + 1) / 2) nq with partial) is the Debye intensity the calc functions returned
 * for ntot atoms; per block, the sinc sum over site pairs closer than each site's farthest neighbour
 * plus Rcorr is removed and the sum over its listed neighbours added (weights ff[e][iq] or sl[e], times
 * coeff), the polarisation factor applied as the reference applies it, and I0 renormalised by the
 * corrected pair count N (which starts from the reference's SQR(Ntot) in unsigned int arithmetic).  With partial the reference accumulates every block into the first block's
 * partial slot; that is kept.  FP64 throughout; terms summed in a different order than the
 * reference's, so within FP64 rounding of it. */
int xns_rearrangement_int(xns_ctx *ctx, double *I0, const double *q, uint32_t nq, const xns_rearr_block *blocks,
                          uint32_t nblocks, uint32_t nel, int source, const double *const *ff, const double *sl,
                          int partial, int polar, double lambda, uint32_t ntot);

/* ---- output writers ---------------------------------------------------------------------------------- */

/* The reference's text outputs, byte for byte, formatted on all host threads (no device needed).
 * Every number is printed as printf's "%.6e", as the reference's ios::scientific streams print it.
 * Each returns 0, or -1 when the file cannot be written.  The file names are the caller's; the
 * reference builds them as <name>_<xray|neut>_<kind>.txt (IO.cpp:55-57, :112-113, :150-151).
 *   xns_write_i      printI (IO.cpp:109-124) and, per block pair, printPartialI (:125-147):
 *                    "q<TAB>I" per q point.
 *   xns_write_i2     printI2 (IO.cpp:148-167): one row per q, nfi values each followed by a TAB.
 *   xns_write_pdf    printPDF (IO.cpp:51-73, partial = 0) and, per element pair, printPartialPDF
 *                    (:74-108, partial = 1): "r<TAB>value" for r = (i + 0.5) bin, rows up to the last
 *                    one whose |value| (total) or value (partial) exceeds 1e-10.
 *   xns_write_atoms  printAtoms (IO.cpp:273-295): Ntot, an empty line, then "name x  y  z" per atom,
 *                    elements in the order given (the reference's ID map order). */
int xns_write_i(const char *path, const double *q, const double *I, uint32_t nq);
int xns_write_i2(const char *path, const double *I2D, uint32_t nq, uint32_t nfi);
int xns_write_pdf(const char *path, const double *pdf, uint32_t nhist, double bin, int partial);
int xns_write_atoms(const char *path, const double *xyz, const uint32_t *n_el, uint32_t nel, const char *const *names);

/* ---- utilities (no reference counterpart) -------------------------------------------------------- */

/* Measured FMA-pipe throughput of this device in TFLOP/s (an FMA counts 2 flops): FP64 when fp64 != 0,
 * FP32 otherwise.  The roofline denominator for the FP64 distance and FP32 sinc kernels. */
int xns_measure_fma_peak(xns_ctx *ctx, int fp64, double *tflops);

/* Measured rate of conflict-free shared-memory atomic increments on this device, in 1e9 per second:
 * the roofline of a shared-memory histogram, which makes one such increment per counted pair. */
int xns_measure_smem_atomic_peak(xns_ctx *ctx, double *gops);

#ifdef __cplusplus
}
#endif
#endif /* XNS_B200_H */
