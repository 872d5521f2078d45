/* Test infrastructure only -- the ORACLE, not the product.
 *
 * An FP64 C restatement of the reference XaNSoNS CPU calc functions (CalcFunctions.cpp), used by
 * tests/ and by bench.py's CPU-baseline leg to check the CUDA library.  Each function cites the
 * reference lines it restates.  It is pinned against the reference's own code compiled from source
 * (oracle/_ref/libxnsref.so, built by oracle/Makefile) and against the committed golden vectors in
 * tests/golden/.  Nothing in the product links or calls this file.
 *
 * Coordinates are one flat array of x y z triples, element-major: element 0's n_el[0] atoms first,
 * in the same order as the reference's ra[0], then element 1's, ...  Element pairs (a <= b) are
 * numbered in the reference's loop order (a outer, b inner), P = nel(nel+1)/2.
 */
#ifndef XNS_ORACLE_H
#define XNS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define XO_NEUTRON 0
#define XO_XRAY 1
#define XO_RDF 0
#define XO_PDF 1
#define XO_RPDF 2

/* calcRotMatrix (CalcFunctions.cpp:46-115): intrinsic rotation for the 12 Euler conventions
 * (XZX=0 ... ZXY=11, typedefs.h:59-70); m is row-major 3x3. */
void xo_rot_matrix(const double euler[3], uint32_t convention, double m[9]);

/* GetHistSize (CalcFunctions.cpp:224-243) and GetAtomicDensity (:204-223). */
uint32_t xo_hist_size(const double *xyz, const uint32_t *n_el, uint32_t nel, double bin);
double xo_atomic_density(const double *xyz, const uint32_t *n_el, uint32_t nel);

/* calcHist (CalcFunctions.cpp:757-809): u64 counts of (unsigned)(|ri - rj| / bin), element pair
 * major.  Returns 0, or -1 when a distance falls beyond nhist (the reference writes out of bounds
 * there; the restatement refuses). */
int xo_hist(const double *xyz, const uint32_t *n_el, uint32_t nel, uint32_t nhist, double bin, uint64_t *hist);

/* calcIntDebye (CalcFunctions.cpp:547-633).  ff: nel rows of nq (X-ray); sl: nel (neutron). */
void xo_int_debye(const double *xyz, const uint32_t *n_el, uint32_t nel, const double *q, uint32_t nq, int source,
                  const double *ff, const double *sl, int polar, double lambda, double *I);

/* calcIntPartialDebye (CalcFunctions.cpp:634-756).  n_el_block[e*nblocks+b]; I: (1+Nparts)*nq, total first. */
void xo_int_partial_debye(const double *xyz, const uint32_t *n_el, uint32_t nel, uint32_t nblocks, const uint32_t *n_el_block,
                          const double *q, uint32_t nq, int source, const double *ff, const double *sl, int polar,
                          double lambda, double *I);

/* calcInt1DHist (CalcFunctions.cpp:810-911). */
void xo_int_1d_hist(const uint64_t *hist, const uint32_t *n_el, uint32_t nel, uint32_t nhist, double bin, const double *q,
                    uint32_t nq, int source, const double *ff, const double *sl, int polar, double lambda, double *I);

/* PDF branch of calcPDFandDebye (CalcFunctions.cpp:919-960); pdf: (1+P)*nhist, total first. */
void xo_pdf(const uint64_t *hist, const uint32_t *n_el, uint32_t nel, uint32_t nhist, double bin, int pdftype, double p0,
            const double *sl, double *pdf);

/* calcInt2D (CalcFunctions.cpp:969-1091).  Euler angles in radians.  I2D: nq x nfi row-major. */
void xo_int_2d(const double *xyz, const uint32_t *n_el, uint32_t nel, const double *q, uint32_t nq, uint32_t nfi,
               const double euler_min[3], const double euler_max[3], const uint32_t euler_n[3], uint32_t convention,
               double lambda, int source, const double *ff, const double *sl, int polar, double *I2D, double *I);

/* Cartesian q-plane (no reference counterpart; the reference's amplitude sum CalcFunctions.cpp:1026-1046
 * evaluated at q = (qx0 + ix*dqx, qy0 + iy*dqy, 0)).  Form factor per element: X-ray
 * f(q) = sum_k a_k exp(-b_k (q/4pi)^2) + c with coef[e*9 + 0..3] = a, [4..7] = b, [8] = c;
 * neutron f = sl[e].  I: nqy rows of nqx, I[iy*nqx+ix] = |A|^2 / Ntot. */
void xo_amp_plane(const double *xyz, const uint32_t *n_el, uint32_t nel, double qx0, double dqx, uint32_t nqx, double qy0,
                  double dqy, uint32_t nqy, int source, const double *coef, const double *sl, double *I);

/* Form factor model used by xo_amp_plane. */
double xo_ff_gauss(const double *coef9, double q);

/* One block as block::calcAtoms reads it (CalcFunctions.cpp:251-392); the same layout as the
 * library's xns_block. */
typedef struct xo_block {
  uint32_t natom, nid, nsymm, ncopy;
  uint32_t ncell[3];
  int32_t cutoff, cutoff_copies, ro_mol;
  const uint32_t *natom_el, *id;
  const double *r_atom, *occ, *dev, *p_symm, *r_symm, *r_copy, *cf;
  double e[3][3];
  double r_mean[3];
  double rcut, rcut_copies, dev_mol;
} xo_block;

/* Philox4x32-10 (Salmon et al., SC 2011): ctr and key as four and two 32-bit words. */
void xo_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* block::calcAtoms (CalcFunctions.cpp:251-392) for each block in turn, in the reference's loop order,
 * with the random draws of the library's builder (Philox4x32-10 keyed by seed, counter = (site or
 * symmetry index, copy-and-cell index low and high words, block << 8 | purpose)) in place of the
 * clock-seeded std::default_random_engine.  Returns a malloc'd element-major x y z array (free with
 * xo_free), n_el[nel] atoms per element, n_all (optional) atoms per block element. */
double *xo_build_atoms(const xo_block *blocks, uint32_t nblocks, uint32_t nel, uint64_t seed, uint32_t *n_el,
                       uint32_t *n_all);
void xo_free(void *p);

/* One block for RearrangementInt; the same layout as the library's xns_rearr_block. */
typedef struct xo_rearr_block {
  uint32_t natom, nid, rearrangement, coeff;
  const uint32_t *natom_el, *id;
  const double *r_atom;
  const uint32_t *neighb_off;
  const double *neighb_r;
  const uint32_t *neighb_id;
  double rcorr;
} xo_rearr_block;

/* RearrangementInt (CalcFunctions.cpp:469-545) in the reference's loop order and grouping.  ff: nel x nq
 * row-major (X-ray) or NULL; sl: nel (neutron).  I0 in / out as the reference's I. */
void xo_rearrangement_int(double *I0, const double *q, uint32_t nq, const xo_rearr_block *blocks, uint32_t nblocks,
                          uint32_t nel, int source, const double *ff, const double *sl, int partial, int polar,
                          double lambda, uint32_t ntot);

#ifdef __cplusplus
}
#endif
#endif
