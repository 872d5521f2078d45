// Exact Debye double sum (replaces calcIntDebye / calcIntPartialDebye, CalcFunctions.cpp:547-756,
// and calcIntDebyeKernel*, CalcFunctionsCUDA.cu:1163-1273):
//
//   I(q) = [ sum_e N_e w_e(q)^2 + 2 sum_{a<=b} w_a(q) w_b(q) sum_{pairs} sin(q r)/(q r + 1e-8) ] / N
//
// Atom pairs are enumerated as tile pairs (DB_TI x DB_TJ atoms) over segment pairs: a segment is the
// atoms of one element in one block, so a tile pair belongs to exactly one (part, element pair)
// class.  Each tile pair becomes a tile of sinc records (r, weight 1) for the shared sinc engine
// (sinc_engine.cuh).  The reference's +1e-8 in the denominator changes a term by a relative
// 1e-8/(q r), below FP32 resolution for q r > 0.1.
#include <string.h>

#include "schedule.cuh"
#include "sinc_engine.cuh"

using namespace xns_sinc;

namespace xns_sinc {
// debye_tc.cu: the pair sums on the integer tensor cores into SLOT_PARTIAL ([grid][ncls][nq], grid in
// *grid_out) and the +1e-8 sums into SLOT_EPS_T; *used false (and nothing queued) when the mesh or the
// distances do not suit it.
int debye_tc(xns_ctx *ctx, const DevCoords &dc, const std::vector<Segment> &sa, const std::vector<Segment> &sb,
             const std::vector<uint32_t> &cls, const std::vector<uint32_t> &same, uint32_t ncls, double q0, double dq,
             uint32_t nq, double rmax, uint32_t shard, uint32_t nshard, bool *used, int *grid_out);
}  // namespace xns_sinc

namespace {

constexpr int DB_TI = 8, DB_TJ = 48;
static_assert(DB_TI * DB_TJ == SE_TILE, "tile pair must fill one record tile");

struct AtomPairSrc {
  const double *X, *Y, *Z;
  const SegPair *sp;
  int nsp;

  __device__ uint32_t cls(unsigned long long w) const {
    int s;
    uint32_t I, J;
    xns_decode_tile(sp, nsp, w, &s, &I, &J);
    return sp[s].cls;
  }

  // stage: 3 * (DB_TI + DB_TJ) doubles
  __device__ int fill(unsigned long long w, PairRec *pr, void *stage, const SincParams &p, uint32_t cls) const {
    double *sxi = (double *)stage, *syi = sxi + DB_TI, *szi = syi + DB_TI;
    double *sxj = szi + DB_TI, *syj = sxj + DB_TJ, *szj = syj + DB_TJ;
    int s;
    uint32_t I, J;
    xns_decode_tile(sp, nsp, w, &s, &I, &J);
    const SegPair g = sp[s];
    const uint32_t ib = I * DB_TI, jb = J * DB_TJ;
    // a "same" entry may name an a-tile past the segment's end (see schedule.cuh): it is empty
    const uint32_t ni = ib < g.na ? min((uint32_t)DB_TI, g.na - ib) : 0u, nj = min((uint32_t)DB_TJ, g.nb - jb);
    const int tid = threadIdx.x;
    if (tid < (int)ni) {
      sxi[tid] = X[g.a0 + ib + tid];
      syi[tid] = Y[g.a0 + ib + tid];
      szi[tid] = Z[g.a0 + ib + tid];
    }
    for (int t = tid - DB_TI; t >= 0 && t < (int)nj; t += SE_THREADS) {
      sxj[t] = X[g.b0 + jb + t];
      syj[t] = Y[g.b0 + jb + t];
      szj[t] = Z[g.b0 + jb + t];
    }
    __syncthreads();
    for (int e = tid; e < SE_TILE; e += SE_THREADS) {
      const uint32_t ii = e / DB_TJ, jj = e % DB_TJ;
      PairRec rec = null_rec();
      if (ii < ni && jj < nj && !(g.same && ib + ii >= jb + jj)) {
        double dx = sxi[ii] - sxj[jj], dy = syi[ii] - syj[jj], dz = szi[ii] - szj[jj];
        double r = sqrt(dx * dx + dy * dy + dz * dz);
        // coincident atoms: sin(q*0)/(q*0 + 1e-8) = 0 in the reference
        if (r > 0) rec = make_rec(p, cls, r, 1.0);
      }
      pr[e] = rec;
    }
    __syncthreads();
    return SE_TILE;
  }
};

}  // namespace

// Debye on device coordinates.  out (device): [total | parts] ((1+nparts)*nq when nblocks > 1).
// shard / nshard: only the tile pairs w with w % nshard == shard, and the self term on shard 0 only, so
// that the outputs of shards 0..nshard-1 add up to the whole (the epilogue is affine in the sums).
// rmax: an upper bound of the pair distances (the bounding-box diagonal), for the +1e-8 histogram.
static int debye_device(xns_ctx *ctx, const DevCoords &dc, uint32_t nblocks, const uint32_t *n_el_block, const double *q,
                        uint32_t nq, const double *d_w, int polar, double lambda, double *d_out, double rmax,
                        uint32_t shard = 0, uint32_t nshard = 1) {
  const uint32_t nel = (uint32_t)dc.n_el.size();
  const uint32_t P = xns_npairs(nel);
  const uint32_t nparts = nblocks * (nblocks + 1) / 2;
  std::vector<uint32_t> seg0((size_t)nel * nblocks);
  for (uint32_t e = 0; e < nel; e++) {
    uint32_t s = dc.off_el[e], sum = 0;
    for (uint32_t u = 0; u < nblocks; u++) {
      seg0[(size_t)e * nblocks + u] = s;
      s += n_el_block[e * nblocks + u];
      sum += n_el_block[e * nblocks + u];
    }
    if (sum != dc.n_el[e]) return xns_fail(ctx, XNS_ERR_ARG, "partial Debye: block atom counts do not add up to n_el");
  }
  // segment pairs in the reference's order (CalcFunctions.cpp:661-690): elements a <= b, blocks
  // (u, v) with v >= u when a == b; part = index of (min(u,v), max(u,v)) (:686).
  std::vector<Segment> sa, sb;
  std::vector<uint32_t> cls, same;
  uint32_t t = 0;
  for (uint32_t a = 0; a < nel; a++)
    for (uint32_t b = a; b < nel; b++, t++)
      for (uint32_t u = 0; u < nblocks; u++)
        for (uint32_t v = 0; v < nblocks; v++) {
          if (a == b && v < u) continue;
          uint32_t lo = std::min(u, v), hi = std::max(u, v);
          uint32_t part = nblocks * lo - lo * (lo + 1) / 2 + hi;
          sa.push_back({seg0[(size_t)a * nblocks + u], n_el_block[a * nblocks + u]});
          sb.push_back({seg0[(size_t)b * nblocks + v], n_el_block[b * nblocks + v]});
          cls.push_back(part * P + t);
          same.push_back(a == b && u == v);
        }
  int st;
  if ((st = xns_stage_begin(ctx, STAGE_DEBYE))) return st;
  {
    double q0 = 0, dq = 0;
    if (ctx->debye_tc && xns_uniform_mesh(q, nq, &q0, &dq)) {
      bool used = false;
      int tgrid = 1;
      if ((st = debye_tc(ctx, dc, sa, sb, cls, same, nparts * P, q0, dq, nq, rmax, shard, nshard, &used, &tgrid)))
        return st;
      if (used) {
        if ((st = sinc_epilogue(ctx, tgrid, nparts * P, nel, nblocks, n_el_block, q, nq, true, q0, dq, d_w, dc.ntot, polar,
                                lambda, d_out, (const double *)ctx->slot_ptr[SLOT_PARTIAL], true, shard == 0,
                                (const double *)ctx->slot_ptr[SLOT_EPS_T])))
          return st;
        return xns_stage_end(ctx, STAGE_DEBYE);
      }
    }
  }
  std::vector<SegPair> sched;
  unsigned long long ntiles = xns_build_schedule(sa, sb, cls, same, DB_TI, DB_TJ, &sched);
  SegPair *d_sp = nullptr;
  if (ntiles && (st = xns_upload_schedule(ctx, sched, &d_sp))) return st;
  double q0 = 0, dq = 0;
  const bool uniform = xns_uniform_mesh(q, nq, &q0, &dq);
  SincParams p{};
  p.q0 = q0;
  p.dq = dq;
  p.nq = nq;
  p.ncls = nparts * P;
  p.ntiles = ntiles;
  p.shard = shard;
  p.nshard = nshard;
  if (!uniform && (st = sinc_upload_q(ctx, q, nq, &p.q))) return st;
  AtomPairSrc src{dc.x, dc.y, dc.z, d_sp, (int)sched.size()};
  int grid = 0;
  if ((st = xns_stage_begin(ctx, STAGE_DEBYE))) return st;  // (again: the sinc engine's stage alone)
  if ((st = run_sinc(ctx, p, src, sizeof(double) * 3 * (DB_TI + DB_TJ), uniform, rmax, &grid))) return st;
  if ((st = sinc_epilogue(ctx, grid, p.ncls, nel, nblocks, n_el_block, q, nq, uniform, q0, dq, d_w, dc.ntot, polar, lambda,
                          d_out, nullptr, true, shard == 0, (const double *)ctx->slot_ptr[SLOT_EPS_T])))
    return st;
  return xns_stage_end(ctx, STAGE_DEBYE);
}

static int debye_host(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel, uint32_t nblocks,
                      const uint32_t *n_el_block, const double *q, uint32_t nq, int source, const double *const *ff,
                      const double *sl, int polar, double lambda, double *I, uint32_t shard = 0, uint32_t nshard = 1) {
  if (!ctx) return XNS_ERR_ARG;
  if (nshard == 0 || shard >= nshard) return xns_fail(ctx, XNS_ERR_ARG, "Debye: shard >= nshard");
  if (!q || !I || nq == 0) return xns_fail(ctx, XNS_ERR_ARG, "Debye: null q / I or nq == 0");
  int st;
  DevCoords dc;
  if ((st = xns_upload_coords(ctx, xyz_el, n_el, nel, &dc))) return st;
  if (dc.ntot == 0) return xns_fail(ctx, XNS_ERR_ARG, "Debye: no atoms");
  double *d_w;
  if ((st = xns_upload_weights(ctx, nel, nq, source, ff, sl, &d_w))) return st;
  const uint32_t nparts = nblocks * (nblocks + 1) / 2;
  const size_t nout = (size_t)(nblocks > 1 ? 1 + nparts : 1) * nq;
  void *d_out;
  if ((st = xns_scratch(ctx, SLOT_OUT, sizeof(double) * nout, &d_out))) return st;
  std::vector<uint32_t> neb_single;
  if (nblocks == 1) {
    neb_single.assign(n_el, n_el + nel);
    n_el_block = neb_single.data();
  }
  // bounding-box diagonal: no pair is farther apart
  double lo[3] = {HUGE_VAL, HUGE_VAL, HUGE_VAL}, hi[3] = {-HUGE_VAL, -HUGE_VAL, -HUGE_VAL};
  for (uint32_t e = 0; e < nel; e++)
    for (uint32_t i = 0; i < n_el[e]; i++)
      for (int k = 0; k < 3; k++) {
        const double v = xyz_el[e][3 * (size_t)i + k];
        if (!(v == v) || v == HUGE_VAL || v == -HUGE_VAL)
          return xns_fail(ctx, XNS_ERR_ARG, "Debye: non-finite coordinate");
        lo[k] = v < lo[k] ? v : lo[k];
        hi[k] = v > hi[k] ? v : hi[k];
      }
  const double rmax = sqrt((hi[0] - lo[0]) * (hi[0] - lo[0]) + (hi[1] - lo[1]) * (hi[1] - lo[1]) +
                           (hi[2] - lo[2]) * (hi[2] - lo[2])) * (1 + 1e-12) + 1e-9;
  if ((st = xns_timer_start(ctx))) return st;
  if ((st = debye_device(ctx, dc, nblocks, n_el_block, q, nq, d_w, polar, lambda, (double *)d_out, rmax, shard, nshard)))
    return st;
  if ((st = xns_timer_stop(ctx))) return st;
  XNS_CUDA(ctx, cudaMemcpyAsync(I, d_out, sizeof(double) * nout, cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XNS_OK;
}

extern "C" int xns_calc_int_debye(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel,
                                  const double *q, uint32_t nq, int source, const double *const *ff, const double *sl,
                                  int polar, double lambda, double *I) {
  return debye_host(ctx, xyz_el, n_el, nel, 1, nullptr, q, nq, source, ff, sl, polar, lambda, I);
}

extern "C" int xns_calc_int_partial_debye(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel,
                                          uint32_t nblocks, const uint32_t *n_el_block, const double *q, uint32_t nq,
                                          int source, const double *const *ff, const double *sl, int polar, double lambda,
                                          double *I) {
  if (!ctx) return XNS_ERR_ARG;
  if (nblocks == 0 || !n_el_block) return xns_fail(ctx, XNS_ERR_ARG, "partial Debye: nblocks == 0 or null n_el_block");
  return debye_host(ctx, xyz_el, n_el, nel, nblocks, nblocks == 1 ? nullptr : n_el_block, q, nq, source, ff, sl, polar,
                    lambda, I);
}

extern "C" int xns_calc_int_debye_shard(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel,
                                        uint32_t nblocks, const uint32_t *n_el_block, const double *q, uint32_t nq,
                                        int source, const double *const *ff, const double *sl, int polar, double lambda,
                                        uint32_t shard, uint32_t nshard, double *I) {
  if (!ctx) return XNS_ERR_ARG;
  if (nblocks == 0 || (nblocks > 1 && !n_el_block))
    return xns_fail(ctx, XNS_ERR_ARG, "Debye shard: nblocks == 0 or null n_el_block");
  return debye_host(ctx, xyz_el, n_el, nel, nblocks, nblocks == 1 ? nullptr : n_el_block, q, nq, source, ff, sl, polar,
                    lambda, I, shard, nshard);
}
