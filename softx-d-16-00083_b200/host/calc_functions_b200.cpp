// Drop-in replacement of the reference's four CPU calc functions (the signatures main.cpp:344-347
// declares and CalcFunctions.cpp:547-1091 defines) on top of the xns_b200 CUDA library.
//
// Link the reference program with this file instead of its CPU calc functions: main.cpp, ReadXML.cpp,
// IO.cpp and tinyxml2.cpp unchanged, CalcFunctions.cpp compiled with -D UseCUDA (which removes exactly
// the four functions below, CalcFunctions.cpp:546-1092), plus this object and libxns_b200.so.  The
// XML inputs, the stdout timing lines and the output files stay those of the reference.
//
// Contract kept from the reference: outputs are allocated here with new[] and freed by main
// (main.cpp:518-524); inputs are borrowed; cfg->Nhist and cfg->p0 are set by the caller
// (CalcFunctions.cpp:403-408); NumOMPthreads is ignored.  On a library error the function prints the
// message and exits with -1 instead of returning a partial result.  The device is the one named by
// the XNS_DEVICE environment variable (default 0).
#include <chrono>
#include <cstdlib>
#include <cstring>

#include "typedefs.h"
#include "xns_b200.h"

namespace {

xns_ctx *context() {
  static xns_ctx *ctx = nullptr;
  if (!ctx) {
    const char *dev = getenv("XNS_DEVICE");
    int st = xns_create(dev ? atoi(dev) : 0, &ctx);
    if (st) {
      cout << "Error: " << xns_status_string(st) << ": " << xns_last_error(ctx) << endl;
      exit(-1);
    }
  }
  return ctx;
}

void check(int st) {
  if (st) {
    cout << "Error: " << xns_status_string(st) << ": " << xns_last_error(context()) << endl;
    exit(-1);
  }
}

// per-element coordinate pointers: vect3d<double> is three packed doubles
vector<const double *> coords(const vector<vect3d<double> > *ra, unsigned int nel) {
  static_assert(sizeof(vect3d<double>) == 3 * sizeof(double), "vect3d<double> must be three packed doubles");
  vector<const double *> p(nel, nullptr);
  for (unsigned int e = 0; e < nel; e++)
    if (ra[e].size()) p[e] = &ra[e][0].x;
  return p;
}

vector<const double *> ff_rows(const config *cfg, const vector<double *> &FF) {
  vector<const double *> p;
  if (cfg->source == xray)
    for (unsigned int e = 0; e < FF.size(); e++) p.push_back(FF[e]);
  return p;
}

float seconds_since(chrono::steady_clock::time_point t1) {
  return chrono::duration_cast<chrono::duration<float> >(chrono::steady_clock::now() - t1).count();
}

}  // namespace

// The shim's context, for the other drop-in objects of the relinked program (interpose.cpp).
xns_ctx *xns_shim_context() { return context(); }

// calcIntDebye, CalcFunctions.cpp:547
void calcIntDebye(double **I, const config *cfg, const unsigned int *NatomEl, const vector<vect3d<double> > *ra,
                  vector<double *> FF, vector<double> SL, const double *q, unsigned int Ntot, int NumOMPthreads) {
  (void)Ntot;
  (void)NumOMPthreads;
  chrono::steady_clock::time_point t1 = chrono::steady_clock::now();
  vector<const double *> xyz = coords(ra, cfg->Nel), ff = ff_rows(cfg, FF);
  *I = new double[cfg->q.N];
  check(xns_calc_int_debye(context(), xyz.data(), NatomEl, cfg->Nel, q, cfg->q.N, cfg->source, ff.empty() ? nullptr : ff.data(),
                           SL.empty() ? nullptr : SL.data(), cfg->PolarFactor, cfg->lambda, *I));
  cout << "1D pattern calculation time: " << seconds_since(t1) << " s" << endl;
}

// calcIntPartialDebye, CalcFunctions.cpp:634
void calcIntPartialDebye(double **I, const config *cfg, const unsigned int *NatomEl, const vector<vect3d<double> > *ra,
                         vector<double *> FF, vector<double> SL, const double *q, const block *Block, unsigned int Ntot,
                         int NumOMPthreads) {
  (void)Ntot;
  (void)NumOMPthreads;
  chrono::steady_clock::time_point t1 = chrono::steady_clock::now();
  vector<const double *> xyz = coords(ra, cfg->Nel), ff = ff_rows(cfg, FF);
  // atoms of element e in block b, as CalcFunctions.cpp:648-659 derives them
  vector<uint32_t> neb((size_t)cfg->Nel * cfg->Nblocks, 0);
  for (unsigned int e = 0; e < cfg->Nel; e++)
    for (unsigned int b = 0; b < cfg->Nblocks; b++)
      for (unsigned int k = 0; k < Block[b].Nid; k++)
        if (Block[b].id[k] == e) {
          neb[(size_t)e * cfg->Nblocks + b] = Block[b].NatomElAll[k];
          break;
        }
  const unsigned int nparts = cfg->Nblocks * (cfg->Nblocks + 1) / 2;
  *I = new double[(size_t)(nparts + 1) * cfg->q.N];
  check(xns_calc_int_partial_debye(context(), xyz.data(), NatomEl, cfg->Nel, cfg->Nblocks, neb.data(), q, cfg->q.N,
                                   cfg->source, ff.empty() ? nullptr : ff.data(), SL.empty() ? nullptr : SL.data(),
                                   cfg->PolarFactor, cfg->lambda, *I));
  cout << "1D pattern calculation time: " << seconds_since(t1) << " s" << endl;
}

// calcPDFandDebye, CalcFunctions.cpp:912
void calcPDFandDebye(double **I, double **PDF, const config *cfg, const unsigned int *NatomEl,
                     const vector<vect3d<double> > *ra, vector<double *> FF, vector<double> SL, const double *q,
                     unsigned int Ntot, int NumOMPthreads) {
  (void)Ntot;
  (void)NumOMPthreads;
  chrono::steady_clock::time_point t1 = chrono::steady_clock::now();
  vector<const double *> xyz = coords(ra, cfg->Nel), ff = ff_rows(cfg, FF);
  const unsigned int P = cfg->Nel * (cfg->Nel + 1) / 2;
  const bool want_pdf = cfg->scenario > Debye_hist;
  const bool want_iq = cfg->scenario == Debye_hist || cfg->scenario == DebyePDF;
  if (want_pdf) *PDF = new double[(size_t)(1 + P) * cfg->Nhist];
  if (want_iq) *I = new double[cfg->q.N];
  check(xns_calc_pdf_and_debye(context(), xyz.data(), NatomEl, cfg->Nel, cfg->Nhist, cfg->hist_bin, cfg->scenario,
                               cfg->PDFtype, cfg->p0, want_iq ? q : nullptr, want_iq ? cfg->q.N : 0, cfg->source,
                               ff.empty() ? nullptr : ff.data(), SL.empty() ? nullptr : SL.data(), cfg->PolarFactor,
                               cfg->lambda, want_iq ? *I : nullptr, want_pdf ? *PDF : nullptr, nullptr));
  cout << "Histogram, PDF and 1D pattern calculation time: " << seconds_since(t1) << " s" << endl;
}

// calcInt2D, CalcFunctions.cpp:969
void calcInt2D(double ***I2D, double **I, const config *cfg, const unsigned int *NatomEl, const vector<vect3d<double> > *ra,
               vector<double *> FF, vector<double> SL, const double *q, unsigned int Ntot, int NumOMPthreads) {
  (void)Ntot;
  (void)NumOMPthreads;
  chrono::steady_clock::time_point t1 = chrono::steady_clock::now();
  vector<const double *> xyz = coords(ra, cfg->Nel), ff = ff_rows(cfg, FF);
  const unsigned int nq = cfg->q.N, nfi = cfg->Nfi;
  vector<double> flat((size_t)nq * nfi);
  *I = new double[nq];
  const double emin[3] = {cfg->Euler.min.x, cfg->Euler.min.y, cfg->Euler.min.z};
  const double emax[3] = {cfg->Euler.max.x, cfg->Euler.max.y, cfg->Euler.max.z};
  const uint32_t en[3] = {cfg->Euler.N.x, cfg->Euler.N.y, cfg->Euler.N.z};
  check(xns_calc_int_2d(context(), xyz.data(), NatomEl, cfg->Nel, q, nq, nfi, emin, emax, en, cfg->EulerConvention,
                        cfg->lambda, cfg->source, ff.empty() ? nullptr : ff.data(), SL.empty() ? nullptr : SL.data(),
                        cfg->PolarFactor, flat.data(), *I));
  *I2D = new double *[nq];
  for (unsigned int iq = 0; iq < nq; iq++) {
    (*I2D)[iq] = new double[nfi];
    memcpy((*I2D)[iq], flat.data() + (size_t)iq * nfi, sizeof(double) * nfi);
  }
  cout << "2D pattern calculation time: " << seconds_since(t1) << " s" << endl;
}

namespace {

// the random seed of this run: XNS_SEED, else the clock (as the reference's generator, CalcFunctions.cpp:259)
uint64_t run_seed() {
  static uint64_t seed = 0;
  static bool set = false;
  if (!set) {
    const char *s = getenv("XNS_SEED");
    seed = s ? strtoull(s, nullptr, 10) : (uint64_t)chrono::system_clock::now().time_since_epoch().count();
    set = true;
  }
  return seed;
}

void build_blocks(block *Block, unsigned int Nblocks, vector<vect3d<double> > *ra, unsigned int Nel, uint64_t seed) {
  static_assert(sizeof(vect3d<double>) == 3 * sizeof(double), "vect3d<double> must be three packed doubles");
  vector<xns_block> xb(Nblocks);
  vector<vector<double> > store(Nblocks);  // pSymm, rSymm, rCopy and cf of each block as flat rows
  for (unsigned int iB = 0; iB < Nblocks; iB++) {
    const block &b = Block[iB];
    xns_block &x = xb[iB];
    memset(&x, 0, sizeof(x));
    x.natom = b.Natom;
    x.nid = b.Nid;
    x.nsymm = b.Nsymm;
    x.ncopy = b.Ncopy;
    x.ncell[0] = b.Ncell.x, x.ncell[1] = b.Ncell.y, x.ncell[2] = b.Ncell.z;
    x.cutoff = b.cutoff, x.cutoff_copies = b.cutoffcopies, x.ro_mol = b.ro_mol;
    x.natom_el = b.NatomEl.empty() ? nullptr : &b.NatomEl[0];
    x.id = b.id;
    x.r_atom = b.Natom ? &b.rAtom[0].x : nullptr;
    x.occ = b.occ;
    x.dev = b.dev;
    vector<double> &f = store[iB];
    for (unsigned int is = 0; is < b.Nsymm; is++)
      for (int k = 0; k < 3; k++) f.insert(f.end(), {b.pSymm[k][is].x, b.pSymm[k][is].y, b.pSymm[k][is].z});
    const size_t o_rs = f.size();
    for (unsigned int is = 0; is < b.Nsymm; is++) f.insert(f.end(), {b.rSymm[is].x, b.rSymm[is].y, b.rSymm[is].z});
    const size_t o_rc = f.size();
    for (unsigned int ic = 0; ic < b.Ncopy; ic++) f.insert(f.end(), {b.rCopy[ic].x, b.rCopy[ic].y, b.rCopy[ic].z});
    const size_t o_cf = f.size();
    for (unsigned int ic = 0; ic < b.Ncopy; ic++)
      for (int k = 0; k < 3; k++) f.insert(f.end(), {b.cf[k][ic].x, b.cf[k][ic].y, b.cf[k][ic].z});
    f.push_back(0.0);  // keeps every offset inside the vector
    x.p_symm = f.data(), x.r_symm = f.data() + o_rs, x.r_copy = f.data() + o_rc, x.cf = f.data() + o_cf;
    for (int k = 0; k < 3; k++) {
      x.e[k][0] = b.e[k].x, x.e[k][1] = b.e[k].y, x.e[k][2] = b.e[k].z;
    }
    x.r_mean[0] = b.rMean.x, x.r_mean[1] = b.rMean.y, x.r_mean[2] = b.rMean.z;
    x.rcut = b.Rcut, x.rcut_copies = b.RcutCopies, x.dev_mol = b.dev_mol;
  }
  vector<uint32_t> n_el(Nel), n_all;
  for (unsigned int iB = 0; iB < Nblocks; iB++) n_all.resize(n_all.size() + Block[iB].Nid);
  const double *dev = nullptr;
  check(xns_build_atoms(context(), xb.data(), Nblocks, Nel, seed, n_el.data(), n_all.empty() ? nullptr : n_all.data(), &dev));
  vector<double *> dst(Nel, nullptr);
  vector<size_t> before(Nel);
  for (unsigned int e = 0; e < Nel; e++) {
    before[e] = ra[e].size();
    ra[e].resize(before[e] + n_el[e]);
    if (n_el[e]) dst[e] = &ra[e][before[e]].x;
  }
  check(xns_copy_atoms(context(), dst.data()));
  for (unsigned int iB = 0, o = 0; iB < Nblocks; iB++) {
    Block[iB].NatomElAll.resize(Block[iB].Nid);
    for (unsigned int k = 0; k < Block[iB].Nid; k++, o++) {
      Block[iB].NatomElAll[k] = n_all[o];
      Block[iB].N += n_all[o];
    }
  }
}

}  // namespace

// block::calcAtoms (CalcFunctions.cpp:251-392) of every block on the GPU, for CalcAndPrintAtoms
// (:397), whose loop `for (iB...) Block[iB].calcAtoms(*ra);` this call replaces: the atoms are appended
// to ra[] per element in the reference's order, and each block's NatomElAll and N are set as
// calcAtoms sets them.  The random draws are Philox4x32-10 keyed by the XNS_SEED environment variable;
// without it the seed comes from the clock, as the reference's generator does (CalcFunctions.cpp:259).
void calcAtomsB200(block *Block, unsigned int Nblocks, vector<vect3d<double> > *ra, unsigned int Nel) {
  build_blocks(Block, Nblocks, ra, Nel, run_seed());
}

// One block, for the relinked program's block::calcAtoms (interpose.cpp): each block of a run gets its
// own key (the run's seed advanced by a Weyl step per block), so equal blocks draw differently.
void xns_shim_build_block(block *b, vector<vect3d<double> > *ra) {
  static uint64_t calls = 0;
  unsigned int nel = 0;
  for (unsigned int k = 0; k < b->Nid; k++) nel = max(nel, b->id[k] + 1);
  build_blocks(b, 1, ra, nel, run_seed() + 0x9E3779B97F4A7C15ull * ++calls);
}
