// Test infrastructure only: a C-ABI harness around the reference's own CPU calc
// functions, compiled from the reference sources where they lie (see oracle/Makefile).
// It is loaded by tests/, by tests/golden/make_golden.py and by bench.py's
// reference arm as the checker / CPU baseline; the product never links it.
//
// Each xnsref_* function marshals flat arrays into the reference's own types
// (vector<vect3d<double>>[Nel], config, block) and calls the reference function
// named in its comment unchanged.  The reference writes timing lines to cout;
// they are swallowed while a call runs.
#include "typedefs.h"
#include <cstdint>
#include <cstring>

int myid = 0, numprocs = 1;  // main.cpp:315 defines these in the reference program

// Reference entry points (CalcFunctions.cpp), declared with their own signatures.
void calcRotMatrix(vect3d<double> *cf0, vect3d<double> *cf1, vect3d<double> *cf2, vect3d<double> euler, unsigned int convention);
unsigned int GetHistSize(const vector<vect3d<double> > *r, unsigned int Nel, double hist_bin);
double GetAtomicDensity(const vector<vect3d<double> > *r, unsigned int Nel, unsigned int Ntot);
void calcIntDebye(double **I, const config *cfg, const unsigned int *NatomEl, const vector<vect3d<double> > *ra, vector<double *> FF, vector<double> SL, const double *q, unsigned int Ntot, int NumOMPthreads);
void calcIntPartialDebye(double **I, const config *cfg, const unsigned int *NatomEl, const vector<vect3d<double> > *ra, vector<double *> FF, vector<double> SL, const double *q, const block *Block, unsigned int Ntot, int NumOMPthreads);
void calcHist(unsigned long long int **rij_hist, const vector<vect3d<double> > *ra, const unsigned int *NatomEl, unsigned int Nel, unsigned int Nhist, double bin, int NumOMPthreads);
void calcInt1DHist(double **I, unsigned long long int *rij_hist, const unsigned int *NatomEl, unsigned int Nel, const config *cfg, vector<double *> FF, vector<double> SL, const double *q, unsigned int Ntot, int NumOMPthreads);
void calcPDFandDebye(double **I, double **PDF, const config *cfg, const unsigned int *NatomEl, const vector<vect3d<double> > *ra, vector<double *> FF, vector<double> SL, const double *q, unsigned int Ntot, int NumOMPthreads);
void RearrangementInt(double *I0, const double *q, const config *cfg, const block *Block, vector<double *> FF, vector<double> SL, unsigned int Ntot);
int printI(const double *I, unsigned int Nq, const double *q, string name, unsigned int source);
int printI2(const double *const *I2D, unsigned int Nq, unsigned int Nfi, string name, unsigned int source);
int printPartialI(const double *I, unsigned int Nq, const double *q, string name, unsigned int source, unsigned int Nblocks);
int printPDF(const double *PDF, unsigned int Nhist, double hist_bin, string name, unsigned int source, unsigned int PDFtype);
int printPartialPDF(const double *PDF, unsigned int Nhist, double hist_bin, string name, unsigned int source, unsigned int PDFtype, unsigned int Nel, map<string, unsigned int> ID);
int printAtoms(const vector<vect3d<double> > *ra, string name, map<string, unsigned int> ID, unsigned int Ntot);
void calcInt2D(double ***I2D, double **I, const config *cfg, const unsigned int *NatomEl, const vector<vect3d<double> > *ra, vector<double *> FF, vector<double> SL, const double *q, unsigned int Ntot, int NumOMPthreads);

namespace {

struct Quiet {  // swallow the reference's cout timing lines for the duration of a call
  std::ostringstream sink;
  std::streambuf *old;
  Quiet() : old(std::cout.rdbuf(sink.rdbuf())) {}
  ~Quiet() { std::cout.rdbuf(old); }
};

// xyz: all atoms, element-major (element 0's atoms first), x y z per atom.
vector<vect3d<double> > *make_ra(const double *xyz, const uint32_t *n_el, uint32_t nel) {
  vector<vect3d<double> > *ra = new vector<vect3d<double> >[nel];
  size_t off = 0;
  for (uint32_t e = 0; e < nel; e++) {
    ra[e].resize(n_el[e]);
    for (uint32_t i = 0; i < n_el[e]; i++, off++) ra[e][i].assign(xyz[3 * off], xyz[3 * off + 1], xyz[3 * off + 2]);
  }
  return ra;
}

uint32_t total(const uint32_t *n_el, uint32_t nel) {
  uint32_t n = 0;
  for (uint32_t e = 0; e < nel; e++) n += n_el[e];
  return n;
}

void base_config(config *cfg, uint32_t nel, const double *q, uint32_t nq, int source, int polar, double lambda) {
  cfg->scenario = Debye;
  cfg->source = (unsigned)source;
  cfg->Nblocks = 1;
  cfg->Nel = nel;
  cfg->Nfi = 1;
  cfg->Nhist = 0;
  cfg->PDFtype = typePDF;
  cfg->EulerConvention = EulerZXZ;
  cfg->lambda = lambda;
  cfg->hist_bin = 0.001;
  cfg->qPDF = 0;
  cfg->p0 = 0;
  cfg->PolarFactor = polar != 0;
  cfg->PrintAtoms = false;
  cfg->PrintPartialPDF = false;
  cfg->calcPartialIntensity = false;
  cfg->rearrangement = false;
  cfg->q.min = nq ? q[0] : 0;
  cfg->q.max = 0;
  cfg->q.N = nq;
  cfg->Euler.min.assign(0, 0, 0);
  cfg->Euler.max.assign(0, 0, 0);
  cfg->Euler.N.assign(1, 1, 1);
}

// ff: nel rows of nq doubles (X-ray); sl: nel doubles (neutron or PDF weights)
void weights(uint32_t nel, uint32_t nq, const double *ff, const double *sl, vector<double *> *FF, vector<double> *SL) {
  if (ff)
    for (uint32_t e = 0; e < nel; e++) FF->push_back(const_cast<double *>(ff + (size_t)e * nq));
  if (sl)
    for (uint32_t e = 0; e < nel; e++) SL->push_back(sl[e]);
}

}  // namespace

extern "C" {

// calcRotMatrix, CalcFunctions.cpp:46-115.  m is row-major 3x3 (rows cf0, cf1, cf2).
void xnsref_rot_matrix(const double *euler, uint32_t convention, double *m) {
  vect3d<double> c0, c1, c2;
  calcRotMatrix(&c0, &c1, &c2, vect3d<double>(euler[0], euler[1], euler[2]), convention);
  const vect3d<double> rows[3] = {c0, c1, c2};
  for (int r = 0; r < 3; r++) {
    m[3 * r] = rows[r].x;
    m[3 * r + 1] = rows[r].y;
    m[3 * r + 2] = rows[r].z;
  }
}

// GetHistSize, CalcFunctions.cpp:224-243
uint32_t xnsref_hist_size(const double *xyz, const uint32_t *n_el, uint32_t nel, double bin) {
  vector<vect3d<double> > *ra = make_ra(xyz, n_el, nel);
  uint32_t n = GetHistSize(ra, nel, bin);
  delete[] ra;
  return n;
}

// GetAtomicDensity, CalcFunctions.cpp:212-223
double xnsref_atomic_density(const double *xyz, const uint32_t *n_el, uint32_t nel) {
  vector<vect3d<double> > *ra = make_ra(xyz, n_el, nel);
  double p0 = GetAtomicDensity(ra, nel, total(n_el, nel));
  delete[] ra;
  return p0;
}

// calcHist, CalcFunctions.cpp:757-809.  hist_out: Nel(Nel+1)/2 * nhist counts.
int xnsref_calc_hist(const double *xyz, const uint32_t *n_el, uint32_t nel, uint32_t nhist, double bin, int threads, uint64_t *hist_out) {
  vector<vect3d<double> > *ra = make_ra(xyz, n_el, nel);
  unsigned long long *h = NULL;
  calcHist(&h, ra, n_el, nel, nhist, bin, threads);
  std::memcpy(hist_out, h, sizeof(uint64_t) * (size_t)(nel * (nel + 1) / 2) * nhist);
  delete[] h;
  delete[] ra;
  return 0;
}

// calcIntDebye, CalcFunctions.cpp:547-633
int xnsref_calc_int_debye(const double *xyz, const uint32_t *n_el, uint32_t nel, const double *q, uint32_t nq, int source,
                          const double *ff, const double *sl, int polar, double lambda, int threads, double *I_out) {
  Quiet quiet;
  vector<vect3d<double> > *ra = make_ra(xyz, n_el, nel);
  config cfg;
  base_config(&cfg, nel, q, nq, source, polar, lambda);
  vector<double *> FF;
  vector<double> SL;
  weights(nel, nq, ff, sl, &FF, &SL);
  double *I = NULL;
  calcIntDebye(&I, &cfg, n_el, ra, FF, SL, q, total(n_el, nel), threads);
  std::memcpy(I_out, I, sizeof(double) * nq);
  delete[] I;
  delete[] ra;
  return 0;
}

// calcIntPartialDebye, CalcFunctions.cpp:634-756.  n_el_block[e*nblocks+b] = atoms of element e in
// block b (ra[e] holds block 0's atoms of e first).  I_out: (1 + nblocks(nblocks+1)/2) * nq.
int xnsref_calc_int_partial_debye(const double *xyz, const uint32_t *n_el, uint32_t nel, uint32_t nblocks, const uint32_t *n_el_block,
                                  const double *q, uint32_t nq, int source, const double *ff, const double *sl, int polar,
                                  double lambda, int threads, double *I_out) {
  Quiet quiet;
  vector<vect3d<double> > *ra = make_ra(xyz, n_el, nel);
  config cfg;
  base_config(&cfg, nel, q, nq, source, polar, lambda);
  cfg.Nblocks = nblocks;
  cfg.calcPartialIntensity = true;
  block *blocks = new block[nblocks];
  for (uint32_t b = 0; b < nblocks; b++) {
    blocks[b].Nid = nel;
    blocks[b].id = new unsigned int[nel];
    blocks[b].NatomElAll.resize(nel);
    for (uint32_t e = 0; e < nel; e++) {
      blocks[b].id[e] = e;
      blocks[b].NatomElAll[e] = n_el_block[e * nblocks + b];
    }
  }
  vector<double *> FF;
  vector<double> SL;
  weights(nel, nq, ff, sl, &FF, &SL);
  double *I = NULL;
  calcIntPartialDebye(&I, &cfg, n_el, ra, FF, SL, q, blocks, total(n_el, nel), threads);
  std::memcpy(I_out, I, sizeof(double) * (size_t)(1 + nblocks * (nblocks + 1) / 2) * nq);
  delete[] I;
  for (uint32_t b = 0; b < nblocks; b++) delete[] blocks[b].id;  // block's destructor frees id only when Natom != 0
  delete[] blocks;
  delete[] ra;
  return 0;
}

// calcInt1DHist, CalcFunctions.cpp:810-911 (the histogram is read, not modified)
int xnsref_calc_int_1d_hist(const uint64_t *hist, const uint32_t *n_el, uint32_t nel, uint32_t nhist, double bin, const double *q,
                            uint32_t nq, int source, const double *ff, const double *sl, int polar, double lambda, int threads,
                            double *I_out) {
  Quiet quiet;
  config cfg;
  base_config(&cfg, nel, q, nq, source, polar, lambda);
  cfg.scenario = Debye_hist;
  cfg.Nhist = nhist;
  cfg.hist_bin = bin;
  vector<double *> FF;
  vector<double> SL;
  weights(nel, nq, ff, sl, &FF, &SL);
  double *I = NULL;
  calcInt1DHist(&I, const_cast<unsigned long long *>(reinterpret_cast<const unsigned long long *>(hist)), n_el, nel, &cfg, FF, SL, q,
                total(n_el, nel), threads);
  std::memcpy(I_out, I, sizeof(double) * nq);
  delete[] I;
  return 0;
}

// calcPDFandDebye, CalcFunctions.cpp:912-968.  scenario: Debye_hist / PDFonly / DebyePDF.
// pdf_out: (1 + Nel(Nel+1)/2) * nhist (total first) when scenario > Debye_hist; I_out: nq when
// scenario is Debye_hist or DebyePDF.
int xnsref_calc_pdf_and_debye(const double *xyz, const uint32_t *n_el, uint32_t nel, uint32_t nhist, double bin, int scenario,
                              int pdftype, double p0, const double *q, uint32_t nq, int source, const double *ff,
                              const double *sl, int polar, double lambda, int threads, double *I_out, double *pdf_out) {
  Quiet quiet;
  vector<vect3d<double> > *ra = make_ra(xyz, n_el, nel);
  config cfg;
  base_config(&cfg, nel, q, nq, source, polar, lambda);
  cfg.scenario = (unsigned)scenario;
  cfg.Nhist = nhist;
  cfg.hist_bin = bin;
  cfg.PDFtype = (unsigned)pdftype;
  cfg.p0 = p0;
  vector<double *> FF;
  vector<double> SL;
  weights(nel, nq, ff, sl, &FF, &SL);
  double *I = NULL, *PDF = NULL;
  calcPDFandDebye(&I, &PDF, &cfg, n_el, ra, FF, SL, q, total(n_el, nel), threads);
  if (I && I_out) std::memcpy(I_out, I, sizeof(double) * nq);
  if (PDF && pdf_out) std::memcpy(pdf_out, PDF, sizeof(double) * (size_t)(1 + nel * (nel + 1) / 2) * nhist);
  delete[] I;
  delete[] PDF;
  delete[] ra;
  return 0;
}

// calcInt2D, CalcFunctions.cpp:969-1091.  euler angles in radians; I2D_out row-major nq x nfi.
int xnsref_calc_int_2d(const double *xyz, const uint32_t *n_el, uint32_t nel, const double *q, uint32_t nq, uint32_t nfi,
                       const double *euler_min, const double *euler_max, const uint32_t *euler_n, uint32_t convention,
                       double lambda, int source, const double *ff, const double *sl, int polar, int threads, double *I2D_out,
                       double *I_out) {
  Quiet quiet;
  vector<vect3d<double> > *ra = make_ra(xyz, n_el, nel);
  config cfg;
  base_config(&cfg, nel, q, nq, source, polar, lambda);
  cfg.scenario = s2D;
  cfg.Nfi = nfi;
  cfg.EulerConvention = convention;
  cfg.Euler.min.assign(euler_min[0], euler_min[1], euler_min[2]);
  cfg.Euler.max.assign(euler_max[0], euler_max[1], euler_max[2]);
  cfg.Euler.N.assign(euler_n[0], euler_n[1], euler_n[2]);
  vector<double *> FF;
  vector<double> SL;
  weights(nel, nq, ff, sl, &FF, &SL);
  double **I2D = NULL, *I = NULL;
  calcInt2D(&I2D, &I, &cfg, n_el, ra, FF, SL, q, total(n_el, nel), threads);
  for (uint32_t iq = 0; iq < nq; iq++) {
    std::memcpy(I2D_out + (size_t)iq * nfi, I2D[iq], sizeof(double) * nfi);
    delete[] I2D[iq];
  }
  delete[] I2D;
  std::memcpy(I_out, I, sizeof(double) * nq);
  delete[] I;
  delete[] ra;
  return 0;
}

// block::calcAtoms, CalcFunctions.cpp:251-392, for each block in turn (as CalcAndPrintAtoms does,
// :397).  The blocks arrive as the library's xns_block (the same layout is declared here) and are
// copied into the reference's own block objects.  Returns a malloc'd element-major x y z array (free
// with xnsref_free); n_el[nel] atoms per element; n_all (optional) the blocks' NatomElAll.  The
// reference seeds its generator from the clock, so only draw-free inputs repeat.
struct xr_block {
  uint32_t natom, nid, nsymm, ncopy;
  uint32_t ncell[3];
  int32_t cutoff, cutoff_copies, ro_mol;
  const uint32_t *natom_el, *id;
  const double *r_atom, *occ, *dev, *p_symm, *r_symm, *r_copy, *cf;
  double e[3][3];
  double r_mean[3];
  double rcut, rcut_copies, dev_mol;
};

void xnsref_free(void *p) { free(p); }

double *xnsref_calc_atoms(const xr_block *blocks, uint32_t nblocks, uint32_t nel, uint32_t *n_el, uint32_t *n_all) {
  vector<vect3d<double> > *ra = new vector<vect3d<double> >[nel];
  uint32_t o_all = 0;
  for (uint32_t ib = 0; ib < nblocks; ib++) {
    const xr_block &x = blocks[ib];
    block b;
    b.Natom = x.natom;
    b.Nsymm = x.nsymm;
    b.Ncopy = x.ncopy;
    b.create();
    b.Nid = x.nid;
    b.id = new unsigned int[x.nid];
    for (uint32_t k = 0; k < x.nid; k++) {
      b.id[k] = x.id[k];
      b.NatomEl.push_back(x.natom_el[k]);
    }
    b.NatomElAll.resize(x.nid);
    for (uint32_t i = 0; i < x.natom; i++) {
      b.rAtom[i].assign(x.r_atom[3 * i], x.r_atom[3 * i + 1], x.r_atom[3 * i + 2]);
      b.occ[i] = x.occ[i];
      b.dev[i] = x.dev[i];
    }
    for (uint32_t s = 0; s < x.nsymm; s++) {
      for (int k = 0; k < 3; k++) b.pSymm[k][s].assign(x.p_symm[9 * s + 3 * k], x.p_symm[9 * s + 3 * k + 1], x.p_symm[9 * s + 3 * k + 2]);
      b.rSymm[s].assign(x.r_symm[3 * s], x.r_symm[3 * s + 1], x.r_symm[3 * s + 2]);
    }
    for (uint32_t c = 0; c < x.ncopy; c++) {
      for (int k = 0; k < 3; k++) b.cf[k][c].assign(x.cf[9 * c + 3 * k], x.cf[9 * c + 3 * k + 1], x.cf[9 * c + 3 * k + 2]);
      b.rCopy[c].assign(x.r_copy[3 * c], x.r_copy[3 * c + 1], x.r_copy[3 * c + 2]);
    }
    for (int k = 0; k < 3; k++) b.e[k].assign(x.e[k][0], x.e[k][1], x.e[k][2]);
    b.Ncell.assign(x.ncell[0], x.ncell[1], x.ncell[2]);
    b.rMean.assign(x.r_mean[0], x.r_mean[1], x.r_mean[2]);
    b.cutoff = x.cutoff != 0;
    b.Rcut = x.rcut;
    b.cutoffcopies = x.cutoff_copies != 0;
    b.RcutCopies = x.rcut_copies;
    b.dev_mol = x.dev_mol;
    b.ro_mol = x.ro_mol != 0;
    if (x.natom) b.calcAtoms(ra);
    for (uint32_t k = 0; k < x.nid; k++)
      if (n_all) n_all[o_all + k] = x.natom ? b.NatomElAll[k] : 0;
    o_all += x.nid;
  }
  size_t tot = 0;
  for (uint32_t e = 0; e < nel; e++) tot += ra[e].size();
  double *xyz = (double *)malloc(24 * (tot ? tot : 1));
  size_t o = 0;
  for (uint32_t e = 0; e < nel; e++) {
    n_el[e] = (uint32_t)ra[e].size();
    for (size_t i = 0; i < ra[e].size(); i++, o++) {
      xyz[3 * o] = ra[e][i].x;
      xyz[3 * o + 1] = ra[e][i].y;
      xyz[3 * o + 2] = ra[e][i].z;
    }
  }
  delete[] ra;
  return xyz;
}

// The reference's writers (IO.cpp:51-167, 273-295), called unchanged; name is the path prefix the
// reference appends its suffixes to.  I2D is nq x nfi row-major; names: nel element names in the
// reference's ID map order.
int xnsref_print_i(const char *name, const double *q, const double *I, uint32_t nq, uint32_t source) {
  return printI(I, nq, q, string(name), source);
}
int xnsref_print_partial_i(const char *name, const double *q, const double *I, uint32_t nq, uint32_t source, uint32_t nblocks) {
  return printPartialI(I, nq, q, string(name), source, nblocks);
}
int xnsref_print_i2(const char *name, const double *I2D, uint32_t nq, uint32_t nfi, uint32_t source) {
  vector<const double *> rows(nq);
  for (uint32_t i = 0; i < nq; i++) rows[i] = I2D + (size_t)i * nfi;
  return printI2(rows.data(), nq, nfi, string(name), source);
}
int xnsref_print_pdf(const char *name, const double *pdf, uint32_t nhist, double bin, uint32_t source, uint32_t pdftype) {
  return printPDF(pdf, nhist, bin, string(name), source, pdftype);
}
static map<string, unsigned int> id_map(const char *const *names, uint32_t nel) {
  map<string, unsigned int> ID;
  for (uint32_t e = 0; e < nel; e++) ID[names[e]] = e;
  return ID;
}
int xnsref_print_partial_pdf(const char *name, const double *pdf, uint32_t nhist, double bin, uint32_t source, uint32_t pdftype,
                             uint32_t nel, const char *const *names) {
  return printPartialPDF(pdf, nhist, bin, string(name), source, pdftype, nel, id_map(names, nel));
}
int xnsref_print_atoms(const char *name, const double *xyz, const uint32_t *n_el, uint32_t nel, const char *const *names) {
  vector<vect3d<double> > *ra = make_ra(xyz, n_el, nel);
  int r = printAtoms(ra, string(name), id_map(names, nel), total(n_el, nel));
  delete[] ra;
  return r;
}

// RearrangementInt, CalcFunctions.cpp:469-545, on reference blocks built from the library's
// xns_rearr_block layout.  ff: nel x nq row-major (X-ray); I0 in / out.
struct xr_rearr_block {
  uint32_t natom, nid, rearrangement, coeff;
  const uint32_t *natom_el, *id;
  const double *r_atom;
  const uint32_t *neighb_off;
  const double *neighb_r;
  const uint32_t *neighb_id;
  double rcorr;
};

int xnsref_rearrangement_int(double *I0, const double *q, uint32_t nq, const xr_rearr_block *blocks, uint32_t nblocks,
                             uint32_t nel, int source, const double *ff, const double *sl, int partial, int polar,
                             double lambda, uint32_t ntot) {
  config cfg;
  base_config(&cfg, nel, q, nq, source, polar, lambda);
  cfg.Nblocks = nblocks;
  cfg.calcPartialIntensity = partial != 0;
  vector<double *> FF;
  vector<double> SL;
  weights(nel, nq, ff, sl, &FF, &SL);
  block *B = new block[nblocks];
  for (uint32_t b = 0; b < nblocks; b++) {
    const xr_rearr_block &x = blocks[b];
    // coeff = Ncopy * Ncell.x * Ncell.y * Ncell.z * Nsymm (:482): carried by Ncopy, the rest 1
    B[b].Natom = x.natom;
    B[b].Nsymm = 1;
    B[b].Ncopy = x.coeff;
    B[b].rearrangement = x.rearrangement != 0;
    B[b].create();
    B[b].Nid = x.nid;
    B[b].id = new unsigned int[x.nid];
    for (uint32_t k = 0; k < x.nid; k++) B[b].id[k] = x.id[k], B[b].NatomEl.push_back(x.natom_el[k]);
    for (uint32_t i = 0; i < x.natom; i++) B[b].rAtom[i].assign(x.r_atom[3 * i], x.r_atom[3 * i + 1], x.r_atom[3 * i + 2]);
    B[b].Rcorr = x.rcorr;
    if (B[b].rearrangement) {
      B[b].idNeighb = new vector<unsigned>[x.natom];
      for (uint32_t i = 0; i < x.natom; i++)
        for (uint32_t k = x.neighb_off[i]; k < x.neighb_off[i + 1]; k++) {
          B[b].rAtomNeighb[i].push_back(vect3d<double>(x.neighb_r[3 * k], x.neighb_r[3 * k + 1], x.neighb_r[3 * k + 2]));
          B[b].idNeighb[i].push_back(x.neighb_id[k]);
        }
    }
  }
  {
    Quiet quiet;
    RearrangementInt(I0, q, &cfg, B, FF, SL, ntot);
  }
  delete[] B;
  return 0;
}

}  // extern "C"
