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

// d_hist receives classes x nhist u64 counts; structure s owns classes [sum_{s'<s} P(nel_s'),
// + P(nel_s)) in the reference's (a outer, b inner) order.
int xns_hist_set(xns_ctx *ctx, const HistSet &hs, uint32_t nhist, double bin, unsigned long long *d_hist);
