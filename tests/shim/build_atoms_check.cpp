// Test program: the drop-in structure builder calcAtomsB200 (softx-d-16-00083_b200/host/
// calc_functions_b200.cpp) against the reference's own block::calcAtoms (CalcFunctions.cpp:251-392),
// both called on the reference's block objects.  Linked with the reference's CalcFunctions.cpp object
// (compiled from its sources by build.py --shim) and the drop-in libraries.  Draw-free blocks (full
// occupancy, no displacement, no molecule rotation) must give the same atoms in the same order, bit for
// bit, and the same NatomElAll and N.  Prints one line per case; exit status 0 when all agree.
#include <cmath>
#include <cstring>

#include "typedefs.h"

int myid = 0, numprocs = 1;  // main.cpp defines these in the reference program
void calcAtomsB200(block *Block, unsigned int Nblocks, vector<vect3d<double> > *ra, unsigned int Nel);

namespace {

struct Site {
  double x, y, z;
};

// a block with the given Cartesian sites (element-sorted), cell, symmetry translations and copies
void make_block(block &b, const vector<Site> &sites, const vector<unsigned> &natom_el, const vector<unsigned> &id,
                const double e[3][3], unsigned ncx, unsigned ncy, unsigned ncz, const vector<Site> &shifts,
                const vector<Site> &copies, double rot_angle, double rcut, double rcut_copies) {
  b.Natom = (unsigned)sites.size();
  b.Nsymm = (unsigned)shifts.size();
  b.Ncopy = (unsigned)copies.size();
  b.create();
  b.Nid = (unsigned)id.size();
  b.id = new unsigned int[b.Nid];
  for (unsigned k = 0; k < b.Nid; k++) b.id[k] = id[k], b.NatomEl.push_back(natom_el[k]);
  b.NatomElAll.resize(b.Nid);
  for (unsigned i = 0; i < b.Natom; i++) b.rAtom[i].assign(sites[i].x, sites[i].y, sites[i].z);
  for (unsigned s = 0; s < b.Nsymm; s++) {
    b.pSymm[0][s].assign(1, 0, 0), b.pSymm[1][s].assign(0, 1, 0), b.pSymm[2][s].assign(0, 0, 1);
    b.rSymm[s].assign(shifts[s].x, shifts[s].y, shifts[s].z);
  }
  for (unsigned c = 0; c < b.Ncopy; c++) {
    const double a = rot_angle * c, ca = cos(a), sa = sin(a);
    b.cf[0][c].assign(ca, -sa, 0), b.cf[1][c].assign(sa, ca, 0), b.cf[2][c].assign(0, 0, 1);
    b.rCopy[c].assign(copies[c].x, copies[c].y, copies[c].z);
  }
  for (int k = 0; k < 3; k++) b.e[k].assign(e[k][0], e[k][1], e[k][2]);
  b.Ncell.assign(ncx, ncy, ncz);
  b.rMean.assign(0.5 * ncx * e[0][0], 0.5 * ncy * e[1][1], 0.5 * ncz * e[2][2]);
  b.cutoff = rcut > 0, b.Rcut = rcut;
  b.cutoffcopies = rcut_copies > 0, b.RcutCopies = rcut_copies;
}

// the same case built into two sets of blocks, one per builder
typedef void (*Maker)(block *);

void rocksalt(block *B) {
  const double a = 5.64, e[3][3] = {{a, 0, 0}, {0, a, 0}, {0, 0, a}};
  const vector<Site> fcc = {{0, 0, 0}, {0, a / 2, a / 2}, {a / 2, 0, a / 2}, {a / 2, a / 2, 0}};
  make_block(B[0], {{0, 0, 0}, {a / 2, 0, 0}}, {1, 1}, {0, 1}, e, 7, 6, 5, fcc, {{0, 0, 0}}, 0.0, 0.0, 0.0);
}

void copies_cutoffs_two_blocks(block *B) {
  const double a = 4.078, e[3][3] = {{a, 0, 0}, {0, a, 0}, {0, 0, a}};
  const vector<Site> fcc = {{0, 0, 0}, {0, a / 2, a / 2}, {a / 2, 0, a / 2}, {a / 2, a / 2, 0}};
  make_block(B[0], {{0, 0, 0}}, {1}, {1}, e, 8, 8, 8, fcc, {{0, 0, 0}, {40, 5, -3}, {-7, 45, 2}}, 0.4, 14.0, 60.0);
  const double e2[3][3] = {{3.1, 0, 0}, {0, 3.1, 0}, {0, 0, 3.1}};
  // two sites 0.3 A apart: merged, the first (occupancy 1) always wins
  make_block(B[1], {{0, 0, 0}, {0.3, 0, 0}, {1.5, 1.5, 1.5}}, {2, 1}, {0, 2}, e2, 4, 3, 2, {{0, 0, 0}}, {{100, 0, 0}},
             0.0, 0.0, 0.0);
}

bool check(const char *name, Maker make, unsigned nblocks, unsigned nel) {
  vector<block> ref(nblocks), gpu(nblocks);
  make(ref.data());
  make(gpu.data());
  vector<vector<vect3d<double> > > rr(nel), rg(nel);
  for (unsigned iB = 0; iB < nblocks; iB++) ref[iB].calcAtoms(rr.data());
  calcAtomsB200(gpu.data(), nblocks, rg.data(), nel);
  bool ok = true;
  size_t n = 0;
  for (unsigned e = 0; e < nel; e++) {
    n += rr[e].size();
    ok = ok && rr[e].size() == rg[e].size() &&
         (rr[e].empty() || !memcmp(&rr[e][0].x, &rg[e][0].x, rr[e].size() * sizeof(vect3d<double>)));
  }
  for (unsigned iB = 0; iB < nblocks; iB++) {
    ok = ok && ref[iB].N == gpu[iB].N;
    for (unsigned k = 0; k < ref[iB].Nid; k++) ok = ok && ref[iB].NatomElAll[k] == gpu[iB].NatomElAll[k];
  }
  cout << name << ": " << n << " atoms " << (ok ? "identical" : "DIFFER") << endl;
  return ok;
}

}  // namespace

int main() {
  bool ok = check("rocksalt 7x6x5 cells", rocksalt, 1, 2);
  ok = check("copies, cut-offs, merged sites, two blocks", copies_cutoffs_two_blocks, 2, 3) && ok;
  return ok ? 0 : 1;
}
