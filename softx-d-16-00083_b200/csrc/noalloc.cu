// Histogram -> I(q) for callers that cannot allocate device memory.
//
// Some callers of this library run where cudaMalloc is off limits: inside a host framework that owns
// all device memory through its own pool or arena (a plugin handed device buffers by its host, an
// embedded or real-time service whose memory budget is fixed at start-up), or code that must not
// synchronise the device the way an allocation can.  xns_int_1d_hist_noalloc serves them: the caller
// passes the histogram and the output as device buffers it already owns, and every intermediate the
// transform needs lives in g_noalloc_scratch, one file-scope device array of XNS_NOALLOC_SCRATCH_BYTES.
// The function calls no cudaMalloc, cudaFree or other allocating routine.
//
// The array is part of the library image, so every GPU that loads the library holds it until the
// process exits.  In host code g_noalloc_scratch is only a host-side stand-in for the device array:
// its device address comes from cudaGetSymbolAddress, looked up once per device (with that device
// current) by the first call on that device; make that first call before any stream capture.  All
// calls share the array and each call leaves its intermediates there: a call clears what must start
// at zero itself, and calls that overlap on the GPU -- on different streams, or issued from several
// host threads -- race on it.
#include <string.h>

#include <mutex>

#include "bin_source.cuh"
#include "sinc_engine.cuh"

using namespace xns_sinc;

namespace {

constexpr size_t NOALLOC_BYTES = XNS_NOALLOC_SCRATCH_BYTES;
constexpr uint32_t NOALLOC_MAX_NEL = XNS_NOALLOC_MAX_ELEMENTS;
constexpr uint32_t NOALLOC_MAX_PAIRS = NOALLOC_MAX_NEL * (NOALLOC_MAX_NEL + 1) / 2;
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

struct DeviceSetup {
  bool ready;
  unsigned char *scratch;  // device address of g_noalloc_scratch on this device
  int num_sms;
  int per_sm_uniform, per_sm_direct;
};
std::mutex g_setup_mutex;
DeviceSetup g_setup[NOALLOC_MAX_DEVICES];

// Small tables the epilogue reads, passed by value and written into the scratch array.
struct Tables {
  uint32_t pair_a[NOALLOC_MAX_PAIRS], pair_b[NOALLOC_MAX_PAIRS], n_el[NOALLOC_MAX_NEL];
  double sl[NOALLOC_MAX_NEL];
  uint32_t nel, nq;
  int fill_weights;  // neutron: weights[e][iq] = sl[e]
};

__global__ void noalloc_tables_kernel(Tables t, uint32_t *tab, double *w) {
  const uint32_t P = t.nel * (t.nel + 1) / 2;
  for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) {
    tab[i] = t.pair_a[i];
    tab[P + i] = t.pair_b[i];
  }
  for (uint32_t i = threadIdx.x; i < t.nel; i += blockDim.x) tab[2 * P + i] = t.n_el[i];
  if (t.fill_weights)
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < t.nel * t.nq; i += gridDim.x * blockDim.x)
      w[i] = t.sl[i / t.nq];
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// The +1e-8 histogram's bins at most (the array holds P * this many doubles).
constexpr uint32_t NOALLOC_EPS_NB = 4096;

template <int M, bool DIRECT>
cudaError_t prepare(int *per_sm) {
  auto kern = sinc_tiles_kernel<M, DIRECT, BinSrc>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sinc_smem_bytes(M, SE_THREADS, 0));
  if (e != cudaSuccess) return e;
  // the widest layout (one FP64 column per thread): a grid sized by it fits every call
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kern, SE_THREADS, sinc_smem_bytes(M, SE_THREADS, 0));
}

// First call on a device: look up the device address of the scratch array (with that device
// current) and the launch limits.
int device_setup(int dev, DeviceSetup *out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  DeviceSetup &s = g_setup[dev];
  if (!s.ready) {
    void *ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return XNS_ERR_CUDA;
    int major = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) return XNS_ERR_CUDA;
    if (major != 10) return XNS_ERR_NODEV;
    if (cudaDeviceGetAttribute(&s.num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return XNS_ERR_CUDA;
    if (prepare<SE_M_UNIFORM, false>(&s.per_sm_uniform) != cudaSuccess) return XNS_ERR_CUDA;
    if (prepare<SE_M_DIRECT, true>(&s.per_sm_direct) != cudaSuccess) return XNS_ERR_CUDA;
    s.scratch = (unsigned char *)ptr;
    s.ready = true;
  }
  *out = s;
  return XNS_OK;
}

}  // namespace

extern "C" int xns_int_1d_hist_noalloc(const uint64_t *hist_dev, const uint32_t *n_el, uint32_t nel, uint32_t nhist,
                                       double bin, const double *q, uint32_t nq, int source, const double *const *ff,
                                       const double *sl, int polar, double lambda, double *I_dev, void *stream) {
  if (!hist_dev || !n_el || !q || !I_dev || nel == 0 || nq == 0 || nhist == 0 || !(bin > 0)) return XNS_ERR_ARG;
  if (source == XNS_XRAY) {
    if (!ff) return XNS_ERR_ARG;
    for (uint32_t e = 0; e < nel; e++)
      if (!ff[e]) return XNS_ERR_ARG;
  } else if (source != XNS_NEUTRON || !sl) {
    return XNS_ERR_ARG;
  }
  if (nel > NOALLOC_MAX_NEL || nq > XNS_NOALLOC_MAX_Q) return XNS_ERR_LIMIT;
  uint32_t ntot = 0;
  for (uint32_t e = 0; e < nel; e++) ntot += n_el[e];
  if (ntot == 0) return XNS_ERR_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) return XNS_ERR_CUDA;
  DeviceSetup ds;
  int st = device_setup(dev, &ds);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;

  const uint32_t P = nel * (nel + 1) / 2;
  double q0 = 0, dq = 0;
  const bool uniform = xns_uniform_mesh(q, nq, &q0, &dq);
  // one lane per M q values, at most SE_THREADS lanes: 8192 q on a uniform mesh, 2048 otherwise
  const int M = uniform ? SE_M_UNIFORM : SE_M_DIRECT;
  const uint32_t chunks = (nq + M - 1) / M;
  int lanes = 1;
  while (lanes < (int)chunks) lanes <<= 1;
  if (lanes > SE_THREADS || (!uniform && nq > XNS_NOALLOC_MAX_Q_NONUNIFORM)) return XNS_ERR_LIMIT;
  // scratch layout: weights [nel][nq] | q mesh [nq] | tables [2P + nel] | +1e-8 histogram [P][nb] |
  // +1e-8 sums [P][nq] | per-CTA partial sums [G][P][nq]
  uint32_t eps_nb;
  double eps_bin;
  eps_layout((double)nhist * bin, NOALLOC_EPS_NB, &eps_nb, &eps_bin);
  const size_t w_off = 0, q_off = align256(w_off + sizeof(double) * nel * nq);
  const size_t t_off = align256(q_off + sizeof(double) * nq), h_off = align256(t_off + sizeof(uint32_t) * (2 * P + nel));
  const size_t e_off = align256(h_off + sizeof(double) * P * eps_nb), p_off = align256(e_off + sizeof(double) * P * nq);
  const size_t per_cta = sizeof(double) * P * nq;
  if (p_off + per_cta > NOALLOC_BYTES) return XNS_ERR_LIMIT;
  const int per_sm = uniform ? ds.per_sm_uniform : ds.per_sm_direct;
  const uint32_t tpp = (nhist + SE_TILE - 1) / SE_TILE;
  const unsigned long long ntiles = (unsigned long long)tpp * P;
  unsigned long long grid = std::min<unsigned long long>(ntiles, (unsigned long long)ds.num_sms * std::max(per_sm, 1));
  grid = std::min<unsigned long long>(grid, (NOALLOC_BYTES - p_off) / per_cta);
  if (grid == 0) grid = 1;
  double *w = (double *)(ds.scratch + w_off), *dqm = (double *)(ds.scratch + q_off), *partial = (double *)(ds.scratch + p_off);
  double *eps_hist = (double *)(ds.scratch + h_off), *eps_t = (double *)(ds.scratch + e_off);
  uint32_t *tab = (uint32_t *)(ds.scratch + t_off);

  Tables t;
  memset(&t, 0, sizeof(t));
  t.nel = nel;
  t.nq = nq;
  uint32_t k = 0;
  for (uint32_t a = 0; a < nel; a++)
    for (uint32_t b = a; b < nel; b++, k++) {
      t.pair_a[k] = a;
      t.pair_b[k] = b;
    }
  for (uint32_t e = 0; e < nel; e++) {
    t.n_el[e] = n_el[e];
    t.sl[e] = source == XNS_NEUTRON ? sl[e] : 0.0;
  }
  t.fill_weights = source == XNS_NEUTRON;
  // what must start at zero: the +1e-8 histogram and sums, the partial sums (the array keeps the
  // previous call's contents; cudaMemsetAsync allocates nothing)
  if (cudaMemsetAsync(eps_hist, 0, e_off - h_off + sizeof(double) * P * nq, s) != cudaSuccess) return XNS_ERR_CUDA;
  if (cudaMemsetAsync(partial, 0, per_cta * grid, s) != cudaSuccess) return XNS_ERR_CUDA;
  noalloc_tables_kernel<<<std::max(1u, std::min(64u, (nel * nq + 255) / 256)), 256, 0, s>>>(t, tab, w);
  if (cudaGetLastError() != cudaSuccess) return XNS_ERR_CUDA;
  if (source == XNS_XRAY)
    for (uint32_t e = 0; e < nel; e++)
      if (cudaMemcpyAsync(w + (size_t)e * nq, ff[e], sizeof(double) * nq, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return XNS_ERR_CUDA;
  if (!uniform && cudaMemcpyAsync(dqm, q, sizeof(double) * nq, cudaMemcpyHostToDevice, s) != cudaSuccess)
    return XNS_ERR_CUDA;

  SincParams p{};
  p.q0 = q0;
  p.dq = dq;
  p.q = dqm;
  p.nq = nq;
  p.ncls = P;
  p.ntiles = ntiles;
  p.partial = partial;
  p.eps_hist = eps_hist;
  p.eps_nb = eps_nb;
  p.eps_inv_bw = 1.0 / eps_bin;
  BinSrc src{(const unsigned long long *)hist_dev, nhist, tpp, bin};
  if (uniform) {
    const size_t smem = sinc_smem_bytes(SE_M_UNIFORM, lanes, 0);
    sinc_tiles_kernel<SE_M_UNIFORM, false, BinSrc><<<(unsigned)grid, SE_THREADS, smem, s>>>(p, src, lanes);
  } else {
    const size_t smem = sinc_smem_bytes(SE_M_DIRECT, lanes, 0);
    sinc_tiles_kernel<SE_M_DIRECT, true, BinSrc><<<(unsigned)grid, SE_THREADS, smem, s>>>(p, src, lanes);
  }
  if (cudaGetLastError() != cudaSuccess) return XNS_ERR_CUDA;
  dim3 eg((nq + 127) / 128, (eps_nb + EPS_RUN - 1) / EPS_RUN, P);
  sinc_eps_kernel<<<eg, 128, 0, s>>>(eps_hist, eps_nb, eps_bin, q0, dq, uniform ? nullptr : dqm, nq, eps_t);
  if (cudaGetLastError() != cudaSuccess) return XNS_ERR_CUDA;
  sinc_epilogue_kernel<<<(nq + 127) / 128, 128, 0, s>>>(partial, (int)grid, P, nel, 1, 1, tab, tab + P, w, tab + 2 * P, q0, dq,
                                                        uniform ? nullptr : dqm, nq, ntot, polar, lambda, 1, 1, eps_t, I_dev);
  if (cudaGetLastError() != cudaSuccess) return XNS_ERR_CUDA;
  return XNS_OK;
}
