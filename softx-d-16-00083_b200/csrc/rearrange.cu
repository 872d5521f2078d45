// Rearrangement correction: RearrangementInt (CalcFunctions.cpp:469-545) on the GPU.
//
// Per block with a Rearrangement file the reference (one host thread, FP64):
//   - for every ordered pair of the block's sites (i, j), i != j, closer than i's farthest listed
//     neighbour plus Rcorr, removes coeff w_a(q) w_b(q) sin(q r)/(q r + 1e-8) from I and coeff from N;
//   - for every listed neighbour of every site adds the same term for the neighbour's distance and
//     element, and coeff to N;
// then applies the polarisation factor and renormalises I0 by the corrected N.
// Here: the pairs and neighbour terms become a list of entries (distance, elements, sign), counted
// and then written by one thread per (i, j) or (i, neighbour); one thread per q sums a chunk of the
// entries (FP64, the reference's expressions) into the block slot with an FP64 atomic; the epilogue
// kernel does the reference's per-q finishing.  Distances use the reference's operation order
// (typedefs.h:128-131) with no contraction, so the pair selection is the reference's exactly.
#include <math.h>

#include <vector>

#include "xns_internal.cuh"

namespace {

struct Entry {
  double r;
  uint32_t a, b;  // global element indices
  int32_t sign;   // -1 pair inside the block, +1 listed neighbour
  uint32_t pad;
};

__device__ __forceinline__ double sq3(double x, double y, double z) {
  return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

struct RBlock {
  const double *r;          // natom x 3
  const uint32_t *gid;      // global element per site
  const uint32_t *noff;     // natom + 1
  const double *nr;         // neighbours x 3
  const uint32_t *nid;      // neighbours
  const double *rmax2;      // per site
  uint32_t natom;
};

// Rmax2 (CalcFunctions.cpp:244-250) + SQR(Rcorr) (:489)
__global__ void rmax2_kernel(RBlock b, double rcorr, double *rmax2) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= b.natom) return;
  double m = 0;
  for (uint32_t k = b.noff[i]; k < b.noff[i + 1]; k++)
    m = fmax(m, sq3(__dsub_rn(b.r[3 * i], b.nr[3 * k]), __dsub_rn(b.r[3 * i + 1], b.nr[3 * k + 1]),
                    __dsub_rn(b.r[3 * i + 2], b.nr[3 * k + 2])));
  rmax2[i] = __dadd_rn(m, __dmul_rn(rcorr, rcorr));
}

// pairs (i, j) with rij2 < rmax2[i] and rij2 > 1e-6 (:490-493); count only when out == nullptr
__global__ void pair_entries_kernel(RBlock b, unsigned long long *count, Entry *out, unsigned long long cap) {
  const unsigned long long n2 = (unsigned long long)b.natom * b.natom;
  for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < n2;
       t += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t i = (uint32_t)(t / b.natom), j = (uint32_t)(t % b.natom);
    const double r2 = sq3(__dsub_rn(b.r[3 * i], b.r[3 * j]), __dsub_rn(b.r[3 * i + 1], b.r[3 * j + 1]),
                          __dsub_rn(b.r[3 * i + 2], b.r[3 * j + 2]));
    if (!(r2 < b.rmax2[i] && r2 > 0.000001)) continue;
    const unsigned long long at = atomicAdd(count, 1ull);
    if (out && at < cap) out[at] = Entry{sqrt(r2), b.gid[i], b.gid[j], -1, 0};
  }
}

// the listed neighbours of every site (:513-531)
__global__ void neighbour_entries_kernel(RBlock b, unsigned long long *count, Entry *out, unsigned long long cap) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= b.natom) return;
  for (uint32_t k = b.noff[i]; k < b.noff[i + 1]; k++) {
    const double r2 = sq3(__dsub_rn(b.r[3 * i], b.nr[3 * k]), __dsub_rn(b.r[3 * i + 1], b.nr[3 * k + 1]),
                          __dsub_rn(b.r[3 * i + 2], b.nr[3 * k + 2]));
    const unsigned long long at = atomicAdd(count, 1ull);
    if (out && at < cap) out[at] = Entry{sqrt(r2), b.gid[i], b.nid[k], +1, 0};
  }
}

constexpr int SUM_Q = 128;        // q points per CTA
constexpr int SUM_CHUNK = 2048;   // entries per CTA

// I[slot + iq] += sum over a chunk of sign * (coeff w_a w_b) sin(q r) / (q r + 1e-8)
__global__ void __launch_bounds__(SUM_Q) sum_entries_kernel(const Entry *__restrict__ e, unsigned long long n,
                                                            const double *__restrict__ q, uint32_t nq,
                                                            const double *__restrict__ w, double coeff,
                                                            double *__restrict__ I) {
  __shared__ Entry se[256];
  const uint32_t iq = blockIdx.x * SUM_Q + threadIdx.x;
  const double qv = iq < nq ? q[iq] : 0.0;
  double acc = 0;
  // chunks blockIdx.y, blockIdx.y + gridDim.y, ...: the grid's y extent is capped at 65535
  for (unsigned long long lo = (unsigned long long)blockIdx.y * SUM_CHUNK; lo < n;
       lo += (unsigned long long)gridDim.y * SUM_CHUNK) {
    const unsigned long long hi = min(n, lo + SUM_CHUNK);
    for (unsigned long long c = lo; c < hi; c += 256) {
      __syncthreads();
      for (uint32_t k = threadIdx.x; k < 256 && c + k < hi; k += SUM_Q) se[k] = e[c + k];
      __syncthreads();
      if (iq < nq) {
        const uint32_t m = (uint32_t)(hi - c < 256 ? hi - c : 256);
        for (uint32_t k = 0; k < m; k++) {
          const double qr = se[k].r * qv;
          const double wt = __dmul_rn(__dmul_rn(coeff, w[(size_t)se[k].a * nq + iq]), w[(size_t)se[k].b * nq + iq]);
          const double t = __ddiv_rn(__dmul_rn(wt, sin(qr)), __dadd_rn(qr, 0.00000001));
          acc = se[k].sign > 0 ? __dadd_rn(acc, t) : __dsub_rn(acc, t);
        }
      }
    }
  }
  if (iq < nq && (unsigned long long)blockIdx.y * SUM_CHUNK < n) atomicAdd(I + iq, acc);
}

// PolarFactor1D (CalcFunctions.cpp:460-468) for one q
__device__ __forceinline__ double polar_factor(double q, double lambda) {
  const double s = __dmul_rn(q, __ddiv_rn(__dmul_rn(lambda, 0.25), XNS_PI));
  const double c = __dsub_rn(1.0, __dmul_rn(2.0, __dmul_rn(s, s)));
  return __dmul_rn(0.5, __dadd_rn(1.0, __dmul_rn(c, c)));
}

// the finishing of :532-543, one thread per q
__global__ void finish_kernel(double *I, double *I0, const double *q, uint32_t nq, uint32_t nblocks, int partial, int polar,
                              double lambda, double ntot, double sqrt_n) {
  const uint32_t iq = blockIdx.x * blockDim.x + threadIdx.x;
  if (iq >= nq) return;
  const double f = polar ? polar_factor(q[iq], lambda) : 1.0;
  if (partial) {
    for (uint32_t b = 0; b < nblocks; b++) {
      const size_t st = (size_t)(b + 1) * nq, st0 = (size_t)nq * (1 + b * (2 * nblocks - b + 1) / 2);
      double v = I[st + iq];
      if (polar) v = __dmul_rn(v, f);
      I[iq] = __dadd_rn(I[iq], v);
      I0[st0 + iq] = __ddiv_rn(__dadd_rn(__dmul_rn(I0[st0 + iq], ntot), v), sqrt_n);
    }
  } else if (polar) {
    I[iq] = __dmul_rn(I[iq], f);
  }
  I0[iq] = __ddiv_rn(__dadd_rn(__dmul_rn(I0[iq], ntot), I[iq]), sqrt_n);
}

#define XNS_RTRY(x)              \
  do {                           \
    int _s = (x);                \
    if (_s != XNS_OK) return _s; \
  } while (0)

// device allocations of one call, freed on the stream when it ends
struct Scratch {
  xns_ctx *ctx;
  std::vector<void *> p;
  explicit Scratch(xns_ctx *c) : ctx(c) {}
  ~Scratch() {
    for (void *x : p) cudaFreeAsync(x, ctx->stream);
  }
  template <class T>
  int get(size_t n, T **out) {
    void *x = nullptr;
    cudaError_t e = cudaMallocAsync(&x, n ? n * sizeof(T) : 16, ctx->stream);
    if (e != cudaSuccess) return xns_cuda_fail(ctx, e, "cudaMallocAsync");
    p.push_back(x);
    *out = (T *)x;
    return XNS_OK;
  }
};

}  // namespace

extern "C" int xns_rearrangement_int(xns_ctx *ctx, double *I0, const double *q, uint32_t nq, const xns_rearr_block *blocks,
                                     uint32_t nblocks, uint32_t nel, int source, const double *const *ff, const double *sl,
                                     int partial, int polar, double lambda, uint32_t ntot) {
  if (!ctx) return XNS_ERR_ARG;
  if (!I0 || !q || nq == 0 || (nblocks && !blocks) || nel == 0)
    return xns_fail(ctx, XNS_ERR_ARG, "rearrangement_int: I0, q, blocks and nel are required");
  for (uint32_t b = 0; b < nblocks; b++) {
    const xns_rearr_block &B = blocks[b];
    if (!B.rearrangement || !B.natom) continue;
    if (!B.natom_el || !B.id || !B.r_atom || !B.neighb_off || B.nid == 0)
      return xns_fail(ctx, XNS_ERR_ARG, "rearrangement_int: a block array is NULL");
    uint64_t s = 0;
    for (uint32_t k = 0; k < B.nid; k++) {
      if (B.id[k] >= nel) return xns_fail(ctx, XNS_ERR_ARG, "rearrangement_int: element id >= nel");
      s += B.natom_el[k];
    }
    if (s != B.natom) return xns_fail(ctx, XNS_ERR_ARG, "rearrangement_int: natom_el does not sum to natom");
    const uint32_t nn = B.neighb_off[B.natom];
    if (nn && (!B.neighb_r || !B.neighb_id)) return xns_fail(ctx, XNS_ERR_ARG, "rearrangement_int: neighbour arrays NULL");
    for (uint32_t k = 0; k < nn; k++)
      if (B.neighb_id[k] >= nel) return xns_fail(ctx, XNS_ERR_ARG, "rearrangement_int: neighbour element id >= nel");
  }
  double *d_w;
  XNS_RTRY(xns_upload_weights(ctx, nel, nq, source, ff, sl, &d_w));
  Scratch sc(ctx);
  cudaStream_t s = ctx->stream;
  const size_t nint = partial ? (size_t)(nblocks + 1) * nq : nq;
  const size_t n0 = partial ? (size_t)nq * (1 + (size_t)nblocks * (nblocks + 1) / 2) : nq;
  double *d_I, *d_I0, *d_q;
  unsigned long long *d_cnt;
  XNS_RTRY(sc.get(nint, &d_I));
  XNS_RTRY(sc.get(n0, &d_I0));
  XNS_RTRY(sc.get(nq, &d_q));
  XNS_RTRY(sc.get(2, &d_cnt));
  XNS_CUDA(ctx, cudaMemsetAsync(d_I, 0, nint * sizeof(double), s));
  XNS_CUDA(ctx, cudaMemcpyAsync(d_I0, I0, n0 * sizeof(double), cudaMemcpyHostToDevice, s));
  XNS_CUDA(ctx, cudaMemcpyAsync(d_q, q, nq * sizeof(double), cudaMemcpyHostToDevice, s));
  XNS_RTRY(xns_timer_start(ctx));
  // N = SQR(Ntot) in the reference's unsigned int arithmetic, then long long (:471)
  long long N = (long long)(unsigned int)(ntot * ntot);
  // every block adds into the first slot: iqST is q.N for all blocks with partial (:478-479)
  double *slot = d_I + (partial ? nq : 0);
  for (uint32_t b = 0; b < nblocks; b++) {
    const xns_rearr_block &B = blocks[b];
    if (!B.rearrangement || !B.natom) continue;
    const uint32_t nn = B.neighb_off[B.natom];
    std::vector<uint32_t> gid(B.natom);
    for (uint32_t k = 0, a = 0; k < B.nid; k++)
      for (uint32_t m = 0; m < B.natom_el[k]; m++) gid[a++] = B.id[k];
    double *d_r, *d_nr, *d_rmax2;
    uint32_t *d_gid, *d_noff, *d_nid;
    XNS_RTRY(sc.get(3 * (size_t)B.natom, &d_r));
    XNS_RTRY(sc.get(3 * (size_t)nn, &d_nr));
    XNS_RTRY(sc.get(B.natom, &d_rmax2));
    XNS_RTRY(sc.get(B.natom, &d_gid));
    XNS_RTRY(sc.get((size_t)B.natom + 1, &d_noff));
    XNS_RTRY(sc.get(nn, &d_nid));
    XNS_CUDA(ctx, cudaMemcpyAsync(d_r, B.r_atom, 24 * (size_t)B.natom, cudaMemcpyHostToDevice, s));
    if (nn) {
      XNS_CUDA(ctx, cudaMemcpyAsync(d_nr, B.neighb_r, 24 * (size_t)nn, cudaMemcpyHostToDevice, s));
      XNS_CUDA(ctx, cudaMemcpyAsync(d_nid, B.neighb_id, 4 * (size_t)nn, cudaMemcpyHostToDevice, s));
    }
    XNS_CUDA(ctx, cudaMemcpyAsync(d_gid, gid.data(), 4 * (size_t)B.natom, cudaMemcpyHostToDevice, s));
    XNS_CUDA(ctx, cudaMemcpyAsync(d_noff, B.neighb_off, 4 * ((size_t)B.natom + 1), cudaMemcpyHostToDevice, s));
    RBlock rb{d_r, d_gid, d_noff, d_nr, d_nid, d_rmax2, B.natom};
    const unsigned tb = (B.natom + 127) / 128;
    rmax2_kernel<<<tb, 128, 0, s>>>(rb, B.rcorr, d_rmax2);
    XNS_LAUNCHED(ctx);
    const unsigned long long n2 = (unsigned long long)B.natom * B.natom;
    const unsigned pgrid = (unsigned)std::min<unsigned long long>((n2 + 255) / 256, (unsigned long long)ctx->num_sms * 16);
    XNS_CUDA(ctx, cudaMemsetAsync(d_cnt, 0, 2 * sizeof(unsigned long long), s));
    pair_entries_kernel<<<pgrid, 256, 0, s>>>(rb, d_cnt, nullptr, 0);
    XNS_LAUNCHED(ctx);
    neighbour_entries_kernel<<<tb, 128, 0, s>>>(rb, d_cnt + 1, nullptr, 0);
    XNS_LAUNCHED(ctx);
    unsigned long long cnt[2];
    XNS_CUDA(ctx, cudaMemcpyAsync(cnt, d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, s));
    XNS_CUDA(ctx, cudaStreamSynchronize(s));
    const unsigned long long ne = cnt[0] + cnt[1];
    N += (long long)B.coeff * ((long long)cnt[1] - (long long)cnt[0]);
    if (!ne) continue;
    Entry *d_e;
    XNS_RTRY(sc.get(ne, &d_e));
    XNS_CUDA(ctx, cudaMemsetAsync(d_cnt, 0, 2 * sizeof(unsigned long long), s));
    pair_entries_kernel<<<pgrid, 256, 0, s>>>(rb, d_cnt, d_e, cnt[0]);
    XNS_LAUNCHED(ctx);
    neighbour_entries_kernel<<<tb, 128, 0, s>>>(rb, d_cnt + 1, d_e + cnt[0], cnt[1]);
    XNS_LAUNCHED(ctx);
    const dim3 g((nq + SUM_Q - 1) / SUM_Q, (unsigned)std::min<unsigned long long>((ne + SUM_CHUNK - 1) / SUM_CHUNK, 65535));
    sum_entries_kernel<<<g, SUM_Q, 0, s>>>(d_e, ne, d_q, nq, d_w, (double)B.coeff, slot);
    XNS_LAUNCHED(ctx);
  }
  finish_kernel<<<(nq + 127) / 128, 128, 0, s>>>(d_I, d_I0, d_q, nq, nblocks, partial, polar, lambda, (double)ntot,
                                                   sqrt((double)N));
  XNS_LAUNCHED(ctx);
  XNS_RTRY(xns_timer_stop(ctx));
  XNS_CUDA(ctx, cudaMemcpyAsync(I0, d_I0, n0 * sizeof(double), cudaMemcpyDeviceToHost, s));
  XNS_CUDA(ctx, cudaStreamSynchronize(s));
  return XNS_OK;
}
