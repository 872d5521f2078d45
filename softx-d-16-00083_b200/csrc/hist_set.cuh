// A set of independent structures whose pair-distance histograms are computed in one pass
// (hist.cu): the bin width and the number of bins are shared, pairs are formed only inside a
// structure, and each (structure, element pair a <= b) is one class with its own nhist counts.
#pragma once
#include "xns_internal.cuh"

// One structure: elements [e0, e0 + nel) of the set's element list.
struct HistStruct {
  uint32_t e0, nel;
};

struct HistSet {
  const double *x, *y, *z;           // device SoA coordinates of all structures
  std::vector<uint32_t> el_off, el_n; // per element: first atom in x/y/z, atom count
  std::vector<HistStruct> st;         // structures in class order
};

// Plan parameters: mean atoms per cell of the spatial sort (sets the tile extent) and the bins of the
// shared-memory window that slides along the distance axis (its privatisation depth).
// shard / nshard: this plan counts only its share of the tile pairs (every nshard-th run of the
// size-sorted run list and every nshard-th wide tile pair); the shares of shards 0..nshard-1 add up to
// the whole histogram exactly.
// w_begin / max_pairs: this plan takes the tile pairs [w_begin, w_begin + max_pairs) of the structure's
// enumeration (0: all of them, fewer than 2^32); the passes of a large structure add into one histogram.
// The deepest window (bins) that fits in shared memory beside the counting warps' stages.
constexpr uint32_t HIST_WIN_MAX = 42 * 1024 + 512;
struct HistTuning {
  uint32_t cell_target = 56;
  uint32_t win = HIST_WIN_MAX;
  uint32_t shard = 0, nshard = 1;
  unsigned long long w_begin = 0, max_pairs = 0;
  bool ordered = false;  // atoms of each cell in input order (same tiles in every pass or shard)
};

// Everything the counting kernels need, built by xns_hist_plan; the buffers it points to live in the
// context's scratch slots until the next plan.
struct HistLaunch {
  alignas(16) unsigned char params[256];  // the kernels' parameter block (hist.cu)
  unsigned long long *hist = nullptr;     // classes x nhist
  size_t hist_words = 0;
  unsigned int *flags = nullptr;          // [0] pairs beyond nhist, [1] run queue
  uint32_t classes = 0, nranges = 0, window_grid = 0, wide = 0;
  size_t window_smem = 0;
  unsigned long long ntp_total = 0;       // tile pairs of the whole structure (all passes)
  bool zero_hist = true;                  // the counting launches clear the histogram first
};

// d_hist receives classes x nhist u64 counts; structure s owns classes [sum_{s'<s} P(nel_s'),
// + P(nel_s)) in the reference's (a outer, b inner) order.  Synchronous.
int xns_hist_set(xns_ctx *ctx, const HistSet &hs, uint32_t nhist, double bin, unsigned long long *d_hist);
// The same in three steps: the plan (spatial sort, tile pairs, runs; synchronises with the host), the
// counting launches (memsets and kernels only: can be captured in a CUDA graph), the range check.
int xns_hist_plan(xns_ctx *ctx, const HistSet &hs, uint32_t nhist, double bin, unsigned long long *d_hist,
                  const HistTuning &tune, HistLaunch *L);
int xns_hist_enqueue(xns_ctx *ctx, const HistLaunch &L);
int xns_hist_check(xns_ctx *ctx, const HistLaunch &L);
// Tile pairs per pass of the one-structure histogram entry points (16 bytes of device memory each).
constexpr unsigned long long XNS_HIST_PASS_PAIRS = 1ull << 28;
// One shard of a structure's histogram on device coordinates (plan, count, check), in passes of at most
// max_pairs tile pairs (0: XNS_HIST_PASS_PAIRS).
int xns_hist_device_shard(xns_ctx *ctx, const DevCoords &dc, uint32_t nhist, double bin, uint32_t shard, uint32_t nshard,
                          unsigned long long *d_hist, unsigned long long max_pairs = 0);
