// Tile-pair schedule over segment pairs: shared by the histogram and Debye kernels.
#pragma once
#include "xns_internal.cuh"

// Segment pairs are flattened into one index space of tile pairs: entry s owns tile pairs
// [tile_begin, tile_begin + count).  Tiles along a hold tile_a atoms, along b tile_b atoms, with
// tile_b a multiple of tile_a.  A "same" entry (pairs i < j of one segment) enumerates the upper
// triangle Ib <= J of tile_b-sized blocks, each split into tile_b/tile_a a-tiles, so the a-tile index
// I = Ib * ratio + sub may point past the segment's end (an empty tile); any other entry enumerates the
// full TA x TB rectangle.
struct Segment {
  uint32_t start, count;
};

// Builds the schedule for pairs of segments (sa[k], sb[k]) with output class cls[k]; returns the
// number of tile pairs.  tile: atoms per tile along each side.
unsigned long long xns_build_schedule(const std::vector<Segment> &sa, const std::vector<Segment> &sb,
                                      const std::vector<uint32_t> &cls, const std::vector<uint32_t> &same, uint32_t tile_a,
                                      uint32_t tile_b, std::vector<SegPair> *out);

// Uploads the schedule to SLOT_SEGPAIRS.
int xns_upload_schedule(xns_ctx *ctx, const std::vector<SegPair> &sp, SegPair **d_sp);

// Tile pair w -> (schedule entry, I, J).  nsp is small (<= a few hundred entries).
__device__ __forceinline__ void xns_decode_tile(const SegPair *__restrict__ sp, int nsp, unsigned long long w, int *s_out,
                                                uint32_t *I, uint32_t *J) {
  int lo = 0, hi = nsp - 1;
  while (lo < hi) {  // last entry with tile_begin <= w
    int mid = (lo + hi + 1) >> 1;
    if (sp[mid].tile_begin <= w) lo = mid;
    else hi = mid - 1;
  }
  *s_out = lo;
  unsigned long long l = w - sp[lo].tile_begin;
  if (sp[lo].same) {
    const uint32_t ratio = sp[lo].ratio;
    const uint32_t sub = (uint32_t)(l % ratio);
    l /= ratio;
    // l -> (Ib <= J): J = floor((sqrt(8l+1)-1)/2), Ib = l - J(J+1)/2
    unsigned long long j = (unsigned long long)((sqrt(8.0 * (double)l + 1.0) - 1.0) * 0.5);
    while (j * (j + 1) / 2 > l) j--;
    while ((j + 1) * (j + 2) / 2 <= l) j++;
    *J = (uint32_t)j;
    *I = (uint32_t)(l - j * (j + 1) / 2) * ratio + sub;
  } else {
    *I = (uint32_t)(l / sp[lo].tb);
    *J = (uint32_t)(l % sp[lo].tb);
  }
}
