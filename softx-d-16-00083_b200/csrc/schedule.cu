#include "schedule.cuh"

unsigned long long xns_build_schedule(const std::vector<Segment> &sa, const std::vector<Segment> &sb,
                                      const std::vector<uint32_t> &cls, const std::vector<uint32_t> &same, uint32_t tile_a,
                                      uint32_t tile_b, std::vector<SegPair> *out) {
  out->clear();
  unsigned long long total = 0;
  for (size_t k = 0; k < sa.size(); k++) {
    if (!sa[k].count || !sb[k].count) continue;
    SegPair p;
    p.a0 = sa[k].start;
    p.na = sa[k].count;
    p.b0 = sb[k].start;
    p.nb = sb[k].count;
    p.cls = cls[k];
    p.same = same[k];
    p.ta = (p.na + tile_a - 1) / tile_a;
    p.tb = (p.nb + tile_b - 1) / tile_b;
    p.ratio = tile_b / tile_a;
    p.pad = 0;
    unsigned long long n = p.same ? (unsigned long long)p.tb * (p.tb + 1) / 2 * p.ratio : (unsigned long long)p.ta * p.tb;
    p.tile_begin = total;
    total += n;
    out->push_back(p);
  }
  return total;
}

int xns_upload_schedule(xns_ctx *ctx, const std::vector<SegPair> &sp, SegPair **d_sp) {
  void *d, *h;
  int st;
  size_t bytes = sizeof(SegPair) * (sp.size() ? sp.size() : 1);
  if ((st = xns_scratch(ctx, SLOT_SEGPAIRS, bytes, &d))) return st;
  if ((st = xns_pinned(ctx, bytes, &h))) return st;
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  memcpy(h, sp.data(), sizeof(SegPair) * sp.size());
  XNS_CUDA(ctx, cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, ctx->stream));
  *d_sp = (SegPair *)d;
  return XNS_OK;
}
