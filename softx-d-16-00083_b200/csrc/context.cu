// Context, scratch memory, coordinate upload and shared host helpers.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cstdio>

#include "xns_internal.cuh"

int xns_fail(xns_ctx *ctx, int status, const std::string &msg) {
  if (ctx) ctx->err = msg;
  return status;
}

int xns_cuda_fail(xns_ctx *ctx, cudaError_t e, const char *what) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
  return xns_fail(ctx, e == cudaErrorMemoryAllocation ? XNS_ERR_NOMEM : XNS_ERR_CUDA, buf);
}

int xns_scratch(xns_ctx *ctx, ScratchSlot slot, size_t bytes, void **out) {
  if (bytes == 0) bytes = 16;
  if (ctx->slot_size[slot] < bytes) {
    size_t sz = bytes + bytes / 8;  // headroom so slowly growing calls do not reallocate each time
    if (ctx->mem_limit) {
      size_t others = 0;
      for (int s = 0; s < SLOT_COUNT; s++)
        if (s != slot) others += ctx->slot_size[s];
      if (others + bytes > ctx->mem_limit) {
        char buf[160];
        snprintf(buf, sizeof(buf), "device scratch of %zu bytes would exceed the context's memory limit of %zu bytes",
                 others + bytes, ctx->mem_limit);
        return xns_fail(ctx, XNS_ERR_NOMEM, buf);
      }
      sz = std::min(sz, ctx->mem_limit - others);
    }
    if (ctx->slot_ptr[slot]) {
      cudaError_t e = cudaFreeAsync(ctx->slot_ptr[slot], ctx->stream);
      if (e != cudaSuccess) return xns_cuda_fail(ctx, e, "cudaFreeAsync");
      ctx->slot_ptr[slot] = nullptr;
      ctx->slot_size[slot] = 0;
    }
    cudaError_t e = cudaMallocAsync(&ctx->slot_ptr[slot], sz, ctx->stream);
    if (e != cudaSuccess) return xns_cuda_fail(ctx, e, "cudaMallocAsync");
    ctx->slot_size[slot] = sz;
  }
  *out = ctx->slot_ptr[slot];
  return XNS_OK;
}

int xns_pinned(xns_ctx *ctx, size_t bytes, void **out) {
  if (ctx->pinned_size < bytes) {
    if (ctx->pinned) {
      cudaStreamSynchronize(ctx->stream);
      cudaFreeHost(ctx->pinned);
      ctx->pinned = nullptr;
      ctx->pinned_size = 0;
    }
    size_t sz = bytes + bytes / 8;
    cudaError_t e = cudaMallocHost(&ctx->pinned, sz);
    if (e != cudaSuccess) return xns_cuda_fail(ctx, e, "cudaMallocHost");
    ctx->pinned_size = sz;
  }
  *out = ctx->pinned;
  return XNS_OK;
}

int xns_timer_start(xns_ctx *ctx) {
  XNS_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
  ctx->stage_mask = 0;
  return XNS_OK;
}

int xns_stage_begin(xns_ctx *ctx, int k) {
  XNS_CUDA(ctx, cudaEventRecord(ctx->ev_stage[2 * k], ctx->stream));
  return XNS_OK;
}

int xns_stage_end(xns_ctx *ctx, int k) {
  XNS_CUDA(ctx, cudaEventRecord(ctx->ev_stage[2 * k + 1], ctx->stream));
  ctx->stage_mask |= 1u << k;
  return XNS_OK;
}

int xns_timer_stop(xns_ctx *ctx) {
  XNS_CUDA(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
  XNS_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
  float ms = 0;
  XNS_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  ctx->last_ms = ms;
  return XNS_OK;
}

bool xns_uniform_mesh(const double *q, uint32_t nq, double *q0, double *dq) {
  *q0 = nq ? q[0] : 0;
  *dq = 0;
  if (nq < 2) return nq == 1;
  double d = (q[nq - 1] - q[0]) / (nq - 1);
  double scale = fmax(fabs(q[0]), fabs(q[nq - 1]));
  for (uint32_t i = 0; i < nq; i++)
    if (fabs(q[i] - (q[0] + i * d)) > 1e-12 * scale) return false;
  if (!(d > 0)) return false;
  *dq = d;
  return true;
}

// x y z triples (AoS) -> SoA
__global__ void aos_to_soa_kernel(const double *__restrict__ aos, uint32_t n, double *__restrict__ x, double *__restrict__ y,
                                  double *__restrict__ z) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] = aos[3 * (size_t)i];
    y[i] = aos[3 * (size_t)i + 1];
    z[i] = aos[3 * (size_t)i + 2];
  }
}

int xns_upload_coords(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel, DevCoords *dc) {
  if (!xyz_el || !n_el || nel == 0) return xns_fail(ctx, XNS_ERR_ARG, "coordinates: null pointer or nel == 0");
  dc->n_el.assign(n_el, n_el + nel);
  dc->off_el.resize(nel);
  uint64_t n = 0;
  for (uint32_t e = 0; e < nel; e++) {
    dc->off_el[e] = (uint32_t)n;
    n += n_el[e];
    if (n_el[e] && !xyz_el[e]) return xns_fail(ctx, XNS_ERR_ARG, "coordinates: null element array");
  }
  if (n >= (1ull << 31)) return xns_fail(ctx, XNS_ERR_ARG, "coordinates: more than 2^31 atoms");
  dc->ntot = (uint32_t)n;
  void *aos, *soa;
  int st;
  if ((st = xns_scratch(ctx, SLOT_COORDS_AOS, sizeof(double) * 3 * (n ? n : 1), &aos))) return st;
  if ((st = xns_scratch(ctx, SLOT_COORDS_SOA, sizeof(double) * 3 * (n ? n : 1), &soa))) return st;
  for (uint32_t e = 0; e < nel; e++)
    if (n_el[e])
      XNS_CUDA(ctx, cudaMemcpyAsync((double *)aos + 3 * (size_t)dc->off_el[e], xyz_el[e], sizeof(double) * 3 * n_el[e],
                                    cudaMemcpyHostToDevice, ctx->stream));
  double *x = (double *)soa;
  dc->x = x;
  dc->y = x + n;
  dc->z = x + 2 * n;
  if (n) {
    int blocks = (int)std::min<uint64_t>((n + 255) / 256, (uint64_t)ctx->num_sms * 8);
    aos_to_soa_kernel<<<blocks, 256, 0, ctx->stream>>>((const double *)aos, (uint32_t)n, x, x + n, x + 2 * n);
    XNS_LAUNCHED(ctx);
  }
  return XNS_OK;
}

int xns_upload_weights(xns_ctx *ctx, uint32_t nel, uint32_t nq, int source, const double *const *ff, const double *sl,
                       double **d_w) {
  void *p, *h;
  int st;
  if (source == XNS_XRAY) {
    if (!ff) return xns_fail(ctx, XNS_ERR_ARG, "X-ray source needs form factors (ff)");
    for (uint32_t e = 0; e < nel; e++)
      if (!ff[e]) return xns_fail(ctx, XNS_ERR_ARG, "X-ray source: null form-factor row");
  } else if (source == XNS_NEUTRON) {
    if (!sl) return xns_fail(ctx, XNS_ERR_ARG, "neutron source needs scattering lengths (sl)");
  } else {
    return xns_fail(ctx, XNS_ERR_ARG, "source must be XNS_NEUTRON or XNS_XRAY");
  }
  size_t bytes = sizeof(double) * (size_t)nel * nq;
  if ((st = xns_scratch(ctx, SLOT_WEIGHTS, bytes, &p))) return st;
  if ((st = xns_pinned(ctx, bytes, &h))) return st;
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // pinned staging may still feed an earlier copy
  double *hw = (double *)h;
  for (uint32_t e = 0; e < nel; e++)
    for (uint32_t iq = 0; iq < nq; iq++) hw[(size_t)e * nq + iq] = source == XNS_XRAY ? ff[e][iq] : sl[e];
  XNS_CUDA(ctx, cudaMemcpyAsync(p, hw, bytes, cudaMemcpyHostToDevice, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *d_w = (double *)p;
  return XNS_OK;
}

extern "C" {

const char *xns_status_string(int status) {
  switch (status) {
    case XNS_OK: return "ok";
    case XNS_ERR_ARG: return "invalid argument";
    case XNS_ERR_CUDA: return "CUDA error";
    case XNS_ERR_NODEV: return "no compute capability 10.x device";
    case XNS_ERR_RANGE: return "pair distance beyond the histogram";
    case XNS_ERR_NOMEM: return "device memory allocation failed";
    case XNS_ERR_LIMIT: return "size beyond the allocation-free entry point's fixed limits";
    default: return "unknown status";
  }
}

int xns_create(int device, xns_ctx **out) {
  if (!out) return XNS_ERR_ARG;
  *out = nullptr;
  xns_ctx *ctx = new xns_ctx();
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    ctx->err = "no CUDA device visible";
    *out = ctx;
    return XNS_ERR_NODEV;
  }
  if (device < 0) cudaGetDevice(&device);
  if (device >= ndev) {
    ctx->err = "device index out of range";
    *out = ctx;
    return XNS_ERR_ARG;
  }
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  *out = ctx;
  if (prop.major != 10) {
    ctx->err = std::string("device ") + prop.name + " is not compute capability 10.x (sm_100a)";
    return XNS_ERR_NODEV;
  }
  ctx->device = device;
  ctx->num_sms = prop.multiProcessorCount;
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return xns_cuda_fail(ctx, e, "cudaSetDevice");
  e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return xns_cuda_fail(ctx, e, "cudaStreamCreate");
  ctx->stream = ctx->own_stream;
  cudaEventCreate(&ctx->ev0);
  cudaEventCreate(&ctx->ev1);
  for (int k = 0; k < 2 * xns_ctx::NSTAGE; k++) cudaEventCreate(&ctx->ev_stage[k]);
  return XNS_OK;
}

void xns_destroy(xns_ctx *ctx) {
  if (!ctx) return;
  xns_batch_release_cache(ctx);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (int s = 0; s < SLOT_COUNT; s++)
    if (ctx->slot_ptr[s]) cudaFree(ctx->slot_ptr[s]);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  for (int k = 0; k < 2 * xns_ctx::NSTAGE; k++)
    if (ctx->ev_stage[k]) cudaEventDestroy(ctx->ev_stage[k]);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
}

const char *xns_last_error(const xns_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int xns_set_stream(xns_ctx *ctx, void *stream) {
  if (!ctx) return XNS_ERR_ARG;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return XNS_OK;
}

int xns_set_memory_limit(xns_ctx *ctx, uint64_t bytes) {
  if (!ctx) return XNS_ERR_ARG;
  size_t held = 0;
  for (int s = 0; s < SLOT_COUNT; s++) held += ctx->slot_size[s];
  if (bytes && held > bytes) {  // start again under the new cap
    for (int s = 0; s < SLOT_COUNT; s++)
      if (ctx->slot_ptr[s]) {
        XNS_CUDA(ctx, cudaFreeAsync(ctx->slot_ptr[s], ctx->stream));
        ctx->slot_ptr[s] = nullptr;
        ctx->slot_size[s] = 0;
      }
    XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    // cached tables that lived in the released slots
    ctx->tc_q.clear();
    ctx->x_q.clear();
    ctx->tc_bin = ctx->x_bin = 0;
    ctx->tc_kt = ctx->x_kt = 0;
    ctx->atoms_n.clear();
  }
  ctx->mem_limit = (size_t)bytes;
  return XNS_OK;
}

int xns_inject_pipeline_stall(xns_ctx *ctx, uint64_t wait_limit_ns) {
  if (!ctx) return XNS_ERR_ARG;
  if (wait_limit_ns == 0 || wait_limit_ns > 2000000000ull)
    return xns_fail(ctx, XNS_ERR_ARG, "inject_pipeline_stall: the wait limit must be in (0, 2 s]");
  ctx->inject_stall_ns = wait_limit_ns;
  return XNS_OK;
}

int xns_debye_tensor_cores(xns_ctx *ctx, int on) {
  if (!ctx) return XNS_ERR_ARG;
  ctx->debye_tc = on != 0;
  return XNS_OK;
}

double xns_last_kernel_ms(const xns_ctx *ctx) { return ctx ? ctx->last_ms : 0; }

uint64_t xns_kernel_launches(const xns_ctx *ctx) { return ctx ? ctx->launches : 0; }

double xns_last_stage_ms(const xns_ctx *ctx, int stage) {
  if (!ctx || stage < 0 || stage >= xns_ctx::NSTAGE || !(ctx->stage_mask & (1u << stage))) return -1.0;
  float ms = -1.f;
  if (cudaEventSynchronize(ctx->ev_stage[2 * stage + 1]) != cudaSuccess) return -1.0;
  if (cudaEventElapsedTime(&ms, ctx->ev_stage[2 * stage], ctx->ev_stage[2 * stage + 1]) != cudaSuccess) return -1.0;
  return ms;
}

}  // extern "C"

// ---- device-resident coordinates -------------------------------------------------------------

int xns_coords_from_device(xns_ctx *ctx, const double *xyz_dev, const uint32_t *n_el, uint32_t nel, DevCoords *dc) {
  if (!xyz_dev || !n_el || nel == 0) return xns_fail(ctx, XNS_ERR_ARG, "coordinates: null pointer or nel == 0");
  dc->n_el.assign(n_el, n_el + nel);
  dc->off_el.resize(nel);
  uint64_t n = 0;
  for (uint32_t e = 0; e < nel; e++) {
    dc->off_el[e] = (uint32_t)n;
    n += n_el[e];
  }
  if (n >= (1ull << 31)) return xns_fail(ctx, XNS_ERR_ARG, "coordinates: more than 2^31 atoms");
  dc->ntot = (uint32_t)n;
  void *soa;
  int st;
  if ((st = xns_scratch(ctx, SLOT_COORDS_SOA, sizeof(double) * 3 * (n ? n : 1), &soa))) return st;
  double *x = (double *)soa;
  dc->x = x;
  dc->y = x + n;
  dc->z = x + 2 * n;
  if (n) {
    int blocks = (int)std::min<uint64_t>((n + 255) / 256, (uint64_t)ctx->num_sms * 8);
    aos_to_soa_kernel<<<blocks, 256, 0, ctx->stream>>>(xyz_dev, (uint32_t)n, x, x + n, x + 2 * n);
    XNS_LAUNCHED(ctx);
  }
  return XNS_OK;
}

// ---- FMA-pipe throughput probe ---------------------------------------------------------------

template <typename T>
__global__ void fma_probe_kernel(T *out, int iters, T a, T b) {
  // 8 independent chains per thread keep the pipe full; the result is stored so nothing is elided
  T x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 16; k++) {
      x0 = x0 * a + b; x1 = x1 * a + b; x2 = x2 * a + b; x3 = x3 * a + b;
      x4 = x4 * a + b; x5 = x5 * a + b; x6 = x6 * a + b; x7 = x7 * a + b;
    }
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}

// Conflict-free shared-memory atomic increments: each warp hits 32 consecutive words, 8 per thread per
// iteration, 1024 threads per CTA.
__global__ void __launch_bounds__(1024) smem_atomic_probe_kernel(unsigned *out, int iters) {
  __shared__ unsigned h[4096];
  for (int i = threadIdx.x; i < 4096; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const unsigned base = ((threadIdx.x >> 5) * 32u) & 4095u, lane = threadIdx.x & 31u;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) atomicAdd(&h[(base + lane + 512u * k) & 4095u], 1u);
  }
  __syncthreads();
  out[blockIdx.x * blockDim.x + threadIdx.x] = h[threadIdx.x & 4095u];
}

extern "C" int xns_measure_smem_atomic_peak(xns_ctx *ctx, double *gops) {
  if (!ctx || !gops) return XNS_ERR_ARG;
  const int threads = 1024, blocks = ctx->num_sms * 2, iters = 2048;
  void *out;
  int st;
  if ((st = xns_scratch(ctx, SLOT_AUX, sizeof(unsigned) * threads * blocks, &out))) return st;
  float best = 1e30f;
  for (int rep = 0; rep < 4; rep++) {
    XNS_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    smem_atomic_probe_kernel<<<blocks, threads, 0, ctx->stream>>>((unsigned *)out, iters);
    XNS_LAUNCHED(ctx);
    XNS_CUDA(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    XNS_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
    float ms;
    XNS_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    if (rep && ms < best) best = ms;
  }
  *gops = 8.0 * iters * (double)threads * blocks / (best * 1e-3) / 1e9;
  return XNS_OK;
}

extern "C" int xns_measure_fma_peak(xns_ctx *ctx, int fp64, double *tflops) {
  if (!ctx || !tflops) return XNS_ERR_ARG;
  const int threads = 256, blocks = ctx->num_sms * 8, iters = fp64 ? 1024 : 4096;
  void *out;
  int st;
  if ((st = xns_scratch(ctx, SLOT_AUX, sizeof(double) * threads * blocks, &out))) return st;
  float best = 1e30f;
  for (int rep = 0; rep < 4; rep++) {
    XNS_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    if (fp64) fma_probe_kernel<double><<<blocks, threads, 0, ctx->stream>>>((double *)out, iters, 0.999999, 1e-7);
    else fma_probe_kernel<float><<<blocks, threads, 0, ctx->stream>>>((float *)out, iters, 0.999999f, 1e-7f);
    XNS_LAUNCHED(ctx);
    XNS_CUDA(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    XNS_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
    float ms;
    XNS_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    if (rep && ms < best) best = ms;  // first launch is a warm-up
  }
  const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
  *tflops = flops / (best * 1e-3) / 1e12;
  return XNS_OK;
}
