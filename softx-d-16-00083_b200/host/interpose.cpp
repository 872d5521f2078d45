// The relinked program's replacements of the reference functions either side of the calc functions,
// with their signatures: block::calcAtoms (CalcFunctions.cpp:251-392), RearrangementInt (:469-545),
// and the writers printI, printPartialI, printI2, printPDF, printPartialPDF and printAtoms
// (IO.cpp:51-167, 273-295).  None of them sits behind a backend macro in the reference, so build.py
// --shim links this object into the program together with the reference's own CalcFunctions and IO
// objects in which exactly these symbols were made weak (objcopy --weaken-symbol): the program's
// calls then reach the definitions here.  File names, messages and return values are the reference's.
#include <cstring>

#include "typedefs.h"
#include "xns_b200.h"

xns_ctx *xns_shim_context();
void xns_shim_build_block(block *b, vector<vect3d<double> > *ra);

int block::calcAtoms(vector<vect3d<double> > *ra) {
  xns_shim_build_block(this, ra);
  return 0;
}

void RearrangementInt(double *I0, const double *q, const config *cfg, const block *Block, vector<double *> FF,
                      vector<double> SL, unsigned int Ntot) {
  vector<xns_rearr_block> rb(cfg->Nblocks);
  vector<vector<uint32_t> > off(cfg->Nblocks), nid(cfg->Nblocks);
  vector<vector<double> > nr(cfg->Nblocks);
  for (unsigned int iB = 0; iB < cfg->Nblocks; iB++) {
    const block &b = Block[iB];
    xns_rearr_block &x = rb[iB];
    memset(&x, 0, sizeof(x));
    x.natom = b.Natom;
    x.nid = b.Nid;
    x.rearrangement = b.rearrangement;
    x.coeff = b.Ncopy * b.Ncell.x * b.Ncell.y * b.Ncell.z * b.Nsymm;  // CalcFunctions.cpp:482
    x.natom_el = b.NatomEl.empty() ? nullptr : &b.NatomEl[0];
    x.id = b.id;
    x.r_atom = b.Natom ? &b.rAtom[0].x : nullptr;
    x.rcorr = b.Rcorr;
    off[iB].assign(1, 0);
    if (b.rearrangement)
      for (unsigned int i = 0; i < b.Natom; i++) {
        for (size_t k = 0; k < b.rAtomNeighb[i].size(); k++) {
          nr[iB].insert(nr[iB].end(), {b.rAtomNeighb[i][k].x, b.rAtomNeighb[i][k].y, b.rAtomNeighb[i][k].z});
          nid[iB].push_back(b.idNeighb[i][k]);
        }
        off[iB].push_back((uint32_t)nid[iB].size());
      }
    else
      off[iB].assign(b.Natom + 1, 0);
    x.neighb_off = off[iB].data();
    x.neighb_r = nr[iB].empty() ? nullptr : nr[iB].data();
    x.neighb_id = nid[iB].empty() ? nullptr : nid[iB].data();
  }
  vector<const double *> ff;
  if (cfg->source == xray)
    for (size_t e = 0; e < FF.size(); e++) ff.push_back(FF[e]);
  const int st = xns_rearrangement_int(xns_shim_context(), I0, q, cfg->q.N, rb.data(), cfg->Nblocks, cfg->Nel,
                                       cfg->source, ff.empty() ? nullptr : ff.data(), SL.empty() ? nullptr : SL.data(),
                                       cfg->calcPartialIntensity, cfg->PolarFactor, cfg->lambda, Ntot);
  if (st) {
    cout << "Error: " << xns_status_string(st) << ": " << xns_last_error(xns_shim_context()) << endl;
    exit(-1);
  }
}

namespace {

int cannot_open(const string &f) {
  cout << "Error: cannot open file " << f << " for writing." << endl;
  return -1;
}

const char *pdf_kind(unsigned int PDFtype) {
  return PDFtype == typeRDF ? "RDF" : PDFtype == typePDF ? "PDF" : PDFtype == typeRPDF ? "rPDF" : "";
}

}  // namespace

int printI(const double *I, unsigned int Nq, const double *q, string name, unsigned int source) {
  const string f = name + (source == xray ? "_xray_1D.txt" : "_neut_1D.txt");
  return xns_write_i(f.c_str(), q, I, Nq) ? cannot_open(f) : 0;
}

int printPartialI(const double *I, unsigned int Nq, const double *q, string name, unsigned int source,
                  unsigned int Nblocks) {
  unsigned int count = 0;
  int error = 0;
  for (unsigned int iB = 0; iB < Nblocks; iB++)
    for (unsigned int jB = iB; jB < Nblocks; jB++, count += Nq) {
      ostringstream f;
      f << name << (source == xray ? "_xray_" : "_neut_") << iB << "-" << jB << "_1D.txt";
      if (xns_write_i(f.str().c_str(), q, I + count, Nq)) error += cannot_open(f.str());
    }
  return error;
}

int printI2(const double *const *I, unsigned int Nq, unsigned int Nfi, string name, unsigned int source) {
  const string f = name + (source == xray ? "_xray_2D.txt" : "_neut_2D.txt");
  vector<double> flat((size_t)Nq * Nfi);
  for (unsigned int iq = 0; iq < Nq; iq++) memcpy(&flat[(size_t)iq * Nfi], I[iq], sizeof(double) * Nfi);
  return xns_write_i2(f.c_str(), flat.data(), Nq, Nfi) ? cannot_open(f) : 0;
}

int printPDF(const double *PDF, unsigned int Nhist, double hist_bin, string name, unsigned int source,
             unsigned int PDFtype) {
  const string f = name + (source == xray ? "_xray_" : "_neut_") + pdf_kind(PDFtype) + ".txt";
  return xns_write_pdf(f.c_str(), PDF, Nhist, hist_bin, 0) ? cannot_open(f) : 0;
}

int printPartialPDF(const double *PDF, unsigned int Nhist, double hist_bin, string name, unsigned int source,
                    unsigned int PDFtype, unsigned int Nel, map<string, unsigned int> ID) {
  unsigned int count = 0;
  int error = 0;
  map<string, unsigned int>::iterator it = ID.begin();
  for (unsigned int iEl = 0; iEl < Nel; iEl++, it++) {
    map<string, unsigned int>::iterator jt = it;
    for (unsigned int jEl = iEl; jEl < Nel; jEl++, count += Nhist, jt++) {
      const string f = name + (source == xray ? "_xray_partial_" : "_neut_partial_") + pdf_kind(PDFtype) + "_" +
                       it->first + "_" + jt->first + ".txt";
      if (xns_write_pdf(f.c_str(), PDF + count, Nhist, hist_bin, 1)) error += cannot_open(f);
    }
  }
  return error;
}

int printAtoms(const vector<vect3d<double> > *ra, string name, map<string, unsigned int> ID, unsigned int Ntot) {
  (void)Ntot;  // the writer counts the atoms it prints, which is Ntot (CalcFunctions.cpp:397-402)
  const string f = name + "_atoms.xyz";
  vector<double> xyz;
  vector<uint32_t> n_el;
  vector<const char *> names;
  map<string, unsigned int>::iterator it = ID.begin();
  for (unsigned int iEl = 0; iEl < ID.size(); iEl++, it++) {
    names.push_back(it->first.c_str());
    n_el.push_back((uint32_t)ra[iEl].size());
    for (size_t i = 0; i < ra[iEl].size(); i++) xyz.insert(xyz.end(), {ra[iEl][i].x, ra[iEl][i].y, ra[iEl][i].z});
  }
  return xns_write_atoms(f.c_str(), xyz.empty() ? nullptr : xyz.data(), n_el.data(), (uint32_t)n_el.size(),
                         names.data())
             ? cannot_open(f)
             : 0;
}
