/* Test infrastructure only -- the ORACLE, not the product.  See xns_oracle.h.
 *
 * FP64 restatement of the reference CPU calc functions.  The arithmetic of every quantity that the
 * reference turns into an integer (the histogram bin index) is written operation by operation in the
 * reference's order and compiled without FMA contraction, so histograms are bit-identical to the
 * reference's.  Floating-point sums are accumulated in a different order than the reference's
 * OpenMP zig-zag schedule, so intensities agree to FP64 rounding (~1e-13 relative), not bit for bit.
 */
#include "xns_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define XO_PI 3.1415926535897932384626433832795028841971693993 /* typedefs.h:73 */

static uint32_t total_atoms(const uint32_t *n_el, uint32_t nel) {
  uint32_t n = 0;
  for (uint32_t e = 0; e < nel; e++) n += n_el[e];
  return n;
}

static size_t el_offset(const uint32_t *n_el, uint32_t e) {
  size_t off = 0;
  for (uint32_t i = 0; i < e; i++) off += n_el[i];
  return off;
}

/* vect3d::mag() of (ri - rj): sqrt(SQR(x) + SQR(y) + SQR(z)), typedefs.h:130 */
static double pair_dist(const double *ri, const double *rj) {
  double dx = ri[0] - rj[0], dy = ri[1] - rj[1], dz = ri[2] - rj[2];
  return sqrt(dx * dx + dy * dy + dz * dz);
}

/* ---- rotation ------------------------------------------------------------------------------- */

static void rot_axis(int axis, double a, double m[9]) {
  double c = cos(a), s = sin(a);
  memset(m, 0, 9 * sizeof(double));
  if (axis == 0) { m[0] = 1; m[4] = c; m[5] = -s; m[7] = s; m[8] = c; }
  if (axis == 1) { m[4] = 1; m[0] = c; m[2] = s; m[6] = -s; m[8] = c; }
  if (axis == 2) { m[8] = 1; m[0] = c; m[1] = -s; m[3] = s; m[4] = c; }
}

static void mat_mul(const double a[9], const double b[9], double out[9]) {
  double t[9];
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) t[3 * r + c] = a[3 * r] * b[c] + a[3 * r + 1] * b[3 + c] + a[3 * r + 2] * b[6 + c];
  memcpy(out, t, sizeof(t));
}

/* calcRotMatrix, CalcFunctions.cpp:46-115: for convention "UVW" (typedefs.h:59-70) the matrix is the
 * intrinsic product R_U(alpha) R_V(beta) R_W(gamma). */
void xo_rot_matrix(const double euler[3], uint32_t convention, double m[9]) {
  static const int axes[12][3] = {{0, 2, 0}, {0, 1, 0}, {1, 0, 1}, {1, 2, 1}, {2, 1, 2}, {2, 0, 2},
                                  {0, 2, 1}, {0, 1, 2}, {1, 0, 2}, {1, 2, 0}, {2, 1, 0}, {2, 0, 1}};
  double r0[9], r1[9], r2[9];
  const int *ax = axes[convention % 12];
  rot_axis(ax[0], euler[0], r0);
  rot_axis(ax[1], euler[1], r1);
  rot_axis(ax[2], euler[2], r2);
  mat_mul(r0, r1, m);
  mat_mul(m, r2, m);
}

/* ---- structure metadata --------------------------------------------------------------------- */

/* GetHistSize, CalcFunctions.cpp:224-243 */
uint32_t xo_hist_size(const double *xyz, const uint32_t *n_el, uint32_t nel, double bin) {
  uint32_t n = total_atoms(n_el, nel);
  if (!n) return 1;
  double mx[3], mn[3];
  for (int k = 0; k < 3; k++) mx[k] = mn[k] = xyz[k];
  for (uint32_t i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) {
      double v = xyz[3 * (size_t)i + k];
      if (mx[k] < v) mx[k] = v;
      if (mn[k] > v) mn[k] = v;
    }
  double d[3] = {mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]};
  return (uint32_t)(sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) / bin) + 1;
}

/* GetCenter / GetEnsembleSize / GetAtomicDensity, CalcFunctions.cpp:197-223 */
double xo_atomic_density(const double *xyz, const uint32_t *n_el, uint32_t nel) {
  uint32_t n = total_atoms(n_el, nel);
  double c[3] = {0, 0, 0};
  for (uint32_t i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) c[k] += xyz[3 * (size_t)i + k];
  for (int k = 0; k < 3; k++) c[k] /= n;
  double rmax = 0;
  for (uint32_t i = 0; i < n; i++) {
    double dx = c[0] - xyz[3 * (size_t)i], dy = c[1] - xyz[3 * (size_t)i + 1], dz = c[2] - xyz[3 * (size_t)i + 2];
    double s = dx * dx + dy * dy + dz * dz;
    if (s > rmax) rmax = s;
  }
  double size = 2. * sqrt(rmax);
  double r2 = (0.33333 * size) * (0.33333 * size);
  uint32_t count = 0;
  for (uint32_t i = 0; i < n; i++) {
    double dx = c[0] - xyz[3 * (size_t)i], dy = c[1] - xyz[3 * (size_t)i + 1], dz = c[2] - xyz[3 * (size_t)i + 2];
    if (dx * dx + dy * dy + dz * dz < r2) count++;
  }
  double r = sqrt(r2);
  return count / (4. / 3. * XO_PI * r * r * r);
}

/* ---- histogram ------------------------------------------------------------------------------ */

/* calcHist, CalcFunctions.cpp:757-809: for a <= b, pairs i<j (a == b) or all (i, j), bin
 * (unsigned int)(rij / bin) with rij from vect3d::mag() in FP64. */
int xo_hist(const double *xyz, const uint32_t *n_el, uint32_t nel, uint32_t nhist, double bin, uint64_t *hist) {
  uint32_t P = nel * (nel + 1) / 2;
  memset(hist, 0, sizeof(uint64_t) * (size_t)P * nhist);
  int bad = 0;
  uint32_t t = 0;
  for (uint32_t a = 0; a < nel; a++) {
    for (uint32_t b = a; b < nel; b++, t++) {
      const double *ra = xyz + 3 * el_offset(n_el, a), *rb = xyz + 3 * el_offset(n_el, b);
      uint64_t *h = hist + (size_t)t * nhist;
      int na = (int)n_el[a];
#pragma omp parallel reduction(| : bad)
      {
        uint64_t *loc = (uint64_t *)calloc(nhist, sizeof(uint64_t));
#pragma omp for schedule(dynamic, 16)
        for (int i = 0; i < na; i++) {
          uint32_t j0 = (a == b) ? (uint32_t)i + 1 : 0;
          for (uint32_t j = j0; j < n_el[b]; j++) {
            double r = pair_dist(ra + 3 * (size_t)i, rb + 3 * (size_t)j);
            double k = r / bin;
            if (!(k < (double)nhist)) { bad = 1; continue; }
            loc[(uint32_t)k] += 1;
          }
        }
#pragma omp critical
        for (uint32_t k = 0; k < nhist; k++) h[k] += loc[k];
        free(loc);
      }
    }
  }
  return bad ? -1 : 0;
}

/* ---- Debye sums ----------------------------------------------------------------------------- */

/* PolarFactor1D, CalcFunctions.cpp:460-468 */
static void polar_1d(double *I, const double *q, double lambda, uint32_t nq) {
  for (uint32_t iq = 0; iq < nq; iq++) {
    double s = q[iq] * (lambda * 0.25 / XO_PI);
    double c2 = 1. - 2. * s * s;
    I[iq] *= 0.5 * (1. + c2 * c2);
  }
}

static double weight(int source, const double *ff, const double *sl, uint32_t nq, uint32_t e, uint32_t iq) {
  return source == XO_XRAY ? ff[(size_t)e * nq + iq] : sl[e];
}

/* Sum over the pairs (i in [i0,i1) of element a, j in element b, j > i when same element) of
 * sin(q r)/(q r + 1e-8), CalcFunctions.cpp:574-583; acc[nq] += result.  jlo/jhi restrict j. */
static void debye_pairs(const double *ra, const double *rb, uint32_t i0, uint32_t i1, uint32_t jlo, uint32_t jhi, int same,
                        const double *q, uint32_t nq, double *acc) {
#pragma omp parallel
  {
    double *loc = (double *)calloc(nq, sizeof(double));
#pragma omp for schedule(dynamic, 4)
    for (int i = (int)i0; i < (int)i1; i++) {
      uint32_t js = jlo;
      if (same && (uint32_t)i + 1 > js) js = (uint32_t)i + 1;
      for (uint32_t j = js; j < jhi; j++) {
        double r = pair_dist(ra + 3 * (size_t)i, rb + 3 * (size_t)j);
        for (uint32_t iq = 0; iq < nq; iq++) {
          double x = r * q[iq];
          loc[iq] += sin(x) / (x + 0.00000001);
        }
      }
    }
#pragma omp critical
    for (uint32_t iq = 0; iq < nq; iq++) acc[iq] += loc[iq];
    free(loc);
  }
}

/* calcIntDebye, CalcFunctions.cpp:547-633 */
void xo_int_debye(const double *xyz, const uint32_t *n_el, uint32_t nel, const double *q, uint32_t nq, int source,
                  const double *ff, const double *sl, int polar, double lambda, double *I) {
  uint32_t ntot = total_atoms(n_el, nel);
  double *s = (double *)malloc(sizeof(double) * nq);
  memset(I, 0, sizeof(double) * nq);
  for (uint32_t a = 0; a < nel; a++)
    for (uint32_t b = a; b < nel; b++) {
      memset(s, 0, sizeof(double) * nq);
      debye_pairs(xyz + 3 * el_offset(n_el, a), xyz + 3 * el_offset(n_el, b), 0, n_el[a], 0, n_el[b], a == b, q, nq, s);
      for (uint32_t iq = 0; iq < nq; iq++)
        I[iq] += s[iq] * weight(source, ff, sl, nq, a, iq) * weight(source, ff, sl, nq, b, iq) * 2.;
    }
  for (uint32_t e = 0; e < nel; e++)
    for (uint32_t iq = 0; iq < nq; iq++) {
      double w = weight(source, ff, sl, nq, e, iq);
      I[iq] += n_el[e] * (w * w);
    }
  for (uint32_t iq = 0; iq < nq; iq++) I[iq] /= ntot;
  if (polar) polar_1d(I, q, lambda, nq);
  free(s);
}

/* calcIntPartialDebye, CalcFunctions.cpp:634-756.  Part index of blocks (u <= v):
 * nblocks*u - u(u+1)/2 + v (:686). */
void xo_int_partial_debye(const double *xyz, const uint32_t *n_el, uint32_t nel, uint32_t nblocks, const uint32_t *n_el_block,
                          const double *q, uint32_t nq, int source, const double *ff, const double *sl, int polar,
                          double lambda, double *I) {
  uint32_t ntot = total_atoms(n_el, nel);
  uint32_t nparts = nblocks * (nblocks + 1) / 2;
  double *s = (double *)malloc(sizeof(double) * nq);
  memset(I, 0, sizeof(double) * (size_t)(nparts + 1) * nq);
  for (uint32_t a = 0; a < nel; a++)
    for (uint32_t b = a; b < nel; b++) {
      const double *ra = xyz + 3 * el_offset(n_el, a), *rb = xyz + 3 * el_offset(n_el, b);
      uint32_t ia = 0;
      for (uint32_t u = 0; u < nblocks; u++) {
        uint32_t na = n_el_block[a * nblocks + u];
        uint32_t jb = 0;
        for (uint32_t v = 0; v < nblocks; v++) {
          uint32_t nb = n_el_block[b * nblocks + v];
          if (a != b || v >= u) {
            uint32_t lo = u < v ? u : v, hi = u < v ? v : u;
            uint32_t part = nblocks * lo - lo * (lo + 1) / 2 + hi;
            memset(s, 0, sizeof(double) * nq);
            debye_pairs(ra, rb, ia, ia + na, jb, jb + nb, a == b, q, nq, s);
            for (uint32_t iq = 0; iq < nq; iq++)
              I[(size_t)(part + 1) * nq + iq] +=
                  s[iq] * weight(source, ff, sl, nq, a, iq) * weight(source, ff, sl, nq, b, iq) * 2.;
          }
          jb += nb;
        }
        ia += na;
      }
    }
  for (uint32_t e = 0; e < nel; e++)
    for (uint32_t u = 0; u < nblocks; u++) {
      uint32_t part = nblocks * u - u * (u + 1) / 2 + u;
      for (uint32_t iq = 0; iq < nq; iq++) {
        double w = weight(source, ff, sl, nq, e, iq);
        I[(size_t)(part + 1) * nq + iq] += n_el_block[e * nblocks + u] * (w * w);
      }
    }
  for (size_t k = nq; k < (size_t)(nparts + 1) * nq; k++) I[k] /= ntot;
  if (polar)
    for (uint32_t p = 1; p <= nparts; p++) polar_1d(I + (size_t)p * nq, q, lambda, nq);
  for (uint32_t p = 1; p <= nparts; p++)
    for (uint32_t iq = 0; iq < nq; iq++) I[iq] += I[(size_t)p * nq + iq];
  free(s);
}

/* calcInt1DHist, CalcFunctions.cpp:810-911: r_k = (k + 0.5) bin, empty bins skipped (:857). */
void xo_int_1d_hist(const uint64_t *hist, const uint32_t *n_el, uint32_t nel, uint32_t nhist, double bin, const double *q,
                    uint32_t nq, int source, const double *ff, const double *sl, int polar, double lambda, double *I) {
  uint32_t ntot = total_atoms(n_el, nel);
  double *s = (double *)malloc(sizeof(double) * nq);
  memset(I, 0, sizeof(double) * nq);
  uint32_t t = 0;
  for (uint32_t a = 0; a < nel; a++)
    for (uint32_t b = a; b < nel; b++, t++) {
      const uint64_t *h = hist + (size_t)t * nhist;
      memset(s, 0, sizeof(double) * nq);
#pragma omp parallel
      {
        double *loc = (double *)calloc(nq, sizeof(double));
#pragma omp for schedule(static)
        for (int k = 0; k < (int)nhist; k++) {
          if (!h[k]) continue;
          double r = ((double)k + 0.5) * bin;
          for (uint32_t iq = 0; iq < nq; iq++) {
            double x = r * q[iq];
            loc[iq] += h[k] * sin(x) / (x + 0.00000001);
          }
        }
#pragma omp critical
        for (uint32_t iq = 0; iq < nq; iq++) s[iq] += loc[iq];
        free(loc);
      }
      for (uint32_t iq = 0; iq < nq; iq++)
        I[iq] += 2. * s[iq] * weight(source, ff, sl, nq, a, iq) * weight(source, ff, sl, nq, b, iq);
    }
  for (uint32_t e = 0; e < nel; e++)
    for (uint32_t iq = 0; iq < nq; iq++) {
      double w = weight(source, ff, sl, nq, e, iq);
      I[iq] += n_el[e] * (w * w);
    }
  for (uint32_t iq = 0; iq < nq; iq++) I[iq] /= ntot;
  if (polar) polar_1d(I, q, lambda, nq);
  free(s);
}

/* PDF branch of calcPDFandDebye, CalcFunctions.cpp:919-960.  As in the reference, the radius of
 * element pair t's bin k is evaluated as (t*nhist + k + 0.5)*bin (the loop variable runs over the
 * concatenated histogram, :939-951); for t = 0 that is the bin centre. */
void xo_pdf(const uint64_t *hist, const uint32_t *n_el, uint32_t nel, uint32_t nhist, double bin, int pdftype, double p0,
            const double *sl, double *pdf) {
  uint32_t ntot = total_atoms(n_el, nel);
  uint32_t P = nel * (nel + 1) / 2;
  memset(pdf, 0, sizeof(double) * (size_t)(1 + P) * nhist);
  double fav2 = 0;
  for (uint32_t e = 0; e < nel; e++) fav2 += sl[e] * n_el[e];
  fav2 /= ntot;
  fav2 *= fav2;
  size_t nstart = 0;
  for (uint32_t a = 0; a < nel; a++)
    for (uint32_t b = a; b < nel; b++, nstart += nhist) {
      double mult, sub, r, mij = sl[a] * sl[b] / fav2;
      for (size_t i = nstart; i < nstart + nhist; i++) {
        switch (pdftype) {
          case XO_RDF:
            mult = 2. / (bin * ntot);
            pdf[nhist + i] = hist[i] * mult;
            break;
          case XO_PDF:
            mult = 0.5 / (XO_PI * bin * p0 * ntot);
            r = (i + 0.5) * bin;
            pdf[nhist + i] = hist[i] * mult / (r * r);
            break;
          default:
            mult = 2. / (bin * ntot);
            sub = (b > a) ? 8. * XO_PI * p0 * (double)n_el[a] * (double)n_el[b] / ((double)ntot * (double)ntot)
                          : 4. * XO_PI * p0 * ((double)n_el[a] * (double)n_el[a]) / ((double)ntot * (double)ntot);
            r = (i + 0.5) * bin;
            pdf[nhist + i] = hist[i] * mult / r - sub * r;
            break;
        }
      }
      for (uint32_t i = 0; i < nhist; i++) pdf[i] += pdf[nhist + nstart + i] * mij;
    }
}

/* ---- 2D ------------------------------------------------------------------------------------- */

/* calcInt2D, CalcFunctions.cpp:969-1091 (including sin(theta) = q lambda/4pi, "costheta" = 1 - sin^2,
 * :999-1002; Euler mesh mid-points, :1007-1018; normalisation, polarisation and phi average, :1066-1076) */
void xo_int_2d(const double *xyz, const uint32_t *n_el, uint32_t nel, const double *q, uint32_t nq, uint32_t nfi,
               const double euler_min[3], const double euler_max[3], const uint32_t euler_n[3], uint32_t convention,
               double lambda, int source, const double *ff, const double *sl, int polar, double *I2D, double *I) {
  uint32_t ntot = total_atoms(n_el, nel);
  double dfi = 2. * XO_PI / nfi;
  double d[3];
  for (int k = 0; k < 3; k++) d[k] = euler_n[k] < 2 ? 0 : (euler_max[k] - euler_min[k]) / euler_n[k];
  memset(I2D, 0, sizeof(double) * (size_t)nq * nfi);
  for (uint32_t ia = 0; ia < euler_n[0]; ia++)
    for (uint32_t ib = 0; ib < euler_n[1]; ib++)
      for (uint32_t ig = 0; ig < euler_n[2]; ig++) {
        double eul[3] = {euler_min[0] + (ia + 0.5) * d[0], euler_min[1] + (ib + 0.5) * d[1], euler_min[2] + (ig + 0.5) * d[2]};
        double m[9];
        xo_rot_matrix(eul, convention, m);
#pragma omp parallel for schedule(dynamic, 1)
        for (int iq = 0; iq < (int)nq; iq++) {
          double st = q[iq] * (lambda * 0.25 / XO_PI), ct = 1. - st * st;
          for (uint32_t ifi = 0; ifi < nfi; ifi++) {
            double v[3] = {ct * cos(ifi * dfi) * q[iq], ct * sin(ifi * dfi) * q[iq], -st * q[iq]};
            /* qv' = R^T qv (CS rows are the columns of R, :1020-1022) */
            double w[3];
            for (int c = 0; c < 3; c++) w[c] = v[0] * m[c] + v[1] * m[3 + c] + v[2] * m[6 + c];
            double Ar = 0, Ai = 0;
            size_t off = 0;
            for (uint32_t e = 0; e < nel; e++) {
              double ar = 0, ai = 0;
              for (uint32_t j = 0; j < n_el[e]; j++, off++) {
                const double *r = xyz + 3 * off;
                double x = w[0] * r[0] + w[1] * r[1] + w[2] * r[2];
                ar += cos(x);
                ai += sin(x);
              }
              double f = weight(source, ff, sl, nq, e, (uint32_t)iq);
              Ar += f * ar;
              Ai += f * ai;
            }
            I2D[(size_t)iq * nfi + ifi] += Ar * Ar + Ai * Ai;
          }
        }
      }
  double norm = 1. / ((double)ntot * euler_n[0] * euler_n[1] * euler_n[2]);
  for (uint32_t iq = 0; iq < nq; iq++) {
    double fac = 1;
    if (polar) {
      double s = q[iq] * (lambda * 0.25 / XO_PI), c2 = 1. - 2. * s * s;
      fac = 0.5 * (1. + c2 * c2);
    }
    double sum = 0;
    for (uint32_t ifi = 0; ifi < nfi; ifi++) {
      double *p = I2D + (size_t)iq * nfi + ifi;
      *p *= norm;
      *p *= fac;
      sum += *p;
    }
    I[iq] = sum / nfi;
  }
}

double xo_ff_gauss(const double *c, double q) {
  double s2 = (q / (4. * XO_PI)) * (q / (4. * XO_PI));
  return c[0] * exp(-c[4] * s2) + c[1] * exp(-c[5] * s2) + c[2] * exp(-c[6] * s2) + c[3] * exp(-c[7] * s2) + c[8];
}

void xo_amp_plane(const double *xyz, const uint32_t *n_el, uint32_t nel, double qx0, double dqx, uint32_t nqx, double qy0,
                  double dqy, uint32_t nqy, int source, const double *coef, const double *sl, double *I) {
  uint32_t ntot = total_atoms(n_el, nel);
#pragma omp parallel for schedule(dynamic, 1)
  for (int iy = 0; iy < (int)nqy; iy++) {
    double qy = qy0 + iy * dqy;
    for (uint32_t ix = 0; ix < nqx; ix++) {
      double qx = qx0 + ix * dqx, qm = sqrt(qx * qx + qy * qy);
      double Ar = 0, Ai = 0;
      size_t off = 0;
      for (uint32_t e = 0; e < nel; e++) {
        double ar = 0, ai = 0;
        for (uint32_t j = 0; j < n_el[e]; j++, off++) {
          double x = qx * xyz[3 * off] + qy * xyz[3 * off + 1];
          ar += cos(x);
          ai += sin(x);
        }
        double f = source == XO_XRAY ? xo_ff_gauss(coef + 9 * e, qm) : sl[e];
        Ar += f * ar;
        Ai += f * ai;
      }
      I[(size_t)iy * nqx + ix] = (Ar * Ar + Ai * Ai) / ntot;
    }
  }
}

/* ---- structure builder ------------------------------------------------------------------------ */

void xo_free(void *p) { free(p); }

void xo_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; r++) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n1 = (uint32_t)p1, n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1,
             n3 = (uint32_t)p0;
    c0 = n0, c1 = n1, c2 = n2, c3 = n3;
  }
  out[0] = c0, out[1] = c1, out[2] = c2, out[3] = c3;
}

enum { XO_P_OCC = 0, XO_P_DISP_ANG = 1, XO_P_DISP_RAD = 2, XO_P_MOL_ANG = 3, XO_P_MOL_RAD = 4, XO_P_ROT_A = 5,
       XO_P_ROT_B = 6 };

typedef struct {
  uint32_t key[2], blk;
} xo_rng;

static void rng_draw(const xo_rng *g, uint32_t item, uint64_t unit, uint32_t purpose, double *u0, double *u1) {
  uint32_t c[4] = {item, (uint32_t)unit, (uint32_t)(unit >> 32), (g->blk << 8) | purpose}, r[4];
  xo_philox(c, g->key, r);
  *u0 = (double)(((uint64_t)r[0] << 21) | (r[1] >> 11)) * 0x1.0p-53;
  *u1 = (double)(((uint64_t)r[2] << 21) | (r[3] >> 11)) * 0x1.0p-53;
}

/* CalcFunctions.cpp:335-340 and :366-370: direction phi = 2 pi U, theta = pi U (as the reference draws
 * it), radius |N(0, dev)|; the normal deviate by Box-Muller from two uniforms */
static void rng_displacement(const xo_rng *g, uint32_t item, uint64_t unit, uint32_t p_ang, uint32_t p_rad, double dev,
                             double d[3]) {
  double uf, ut, ua, ub;
  rng_draw(g, item, unit, p_ang, &uf, &ut);
  rng_draw(g, item, unit, p_rad, &ua, &ub);
  double fi = 2.0 * XO_PI * uf, theta = XO_PI * ut;
  double n = sqrt(-2.0 * log(1.0 - ua)) * cos(2.0 * XO_PI * ub);
  double R = fabs(dev * n);
  d[0] = R * sin(theta) * cos(fi);
  d[1] = R * sin(theta) * sin(fi);
  d[2] = R * cos(theta);
}

static double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

typedef struct {
  double *xyz;
  size_t n, cap;
} xo_list;

static void list_push(xo_list *l, const double r[3]) {
  if (l->n == l->cap) {
    l->cap = l->cap ? 2 * l->cap : 1024;
    l->xyz = (double *)realloc(l->xyz, 3 * l->cap * sizeof(double));
  }
  memcpy(l->xyz + 3 * l->n, r, 3 * sizeof(double));
  l->n++;
}

/* one block, appending to the per-element lists (CalcFunctions.cpp:251-392) */
static void build_block(const xo_block *b, uint32_t blk, uint64_t seed, xo_list *out, uint32_t *n_all) {
  const uint32_t S = b->natom * b->nsymm;
  xo_rng g = {{(uint32_t)seed, (uint32_t)(seed >> 32)}, blk};
  double *ra0 = (double *)malloc(3 * (size_t)S * sizeof(double)), *cell = (double *)malloc(3 * (size_t)S * sizeof(double));
  uint32_t *type = (uint32_t *)malloc((size_t)S * sizeof(uint32_t));
  /* :268-274, site order iAtom * Nsymm + iSymm */
  for (uint32_t ia = 0, it = 0, end = b->natom_el[0]; ia < b->natom; ia++) {
    while (ia >= end) end += b->natom_el[++it];
    for (uint32_t is = 0; is < b->nsymm; is++) {
      const uint32_t s = ia * b->nsymm + is;
      const double *p = b->p_symm + 9 * is, *r = b->r_atom + 3 * ia;
      for (int k = 0; k < 3; k++) {
        ra0[3 * s + k] = dot3(p + 3 * k, r);
        cell[3 * s + k] = ra0[3 * s + k] + b->r_symm[3 * is + k];
      }
      type[s] = it;
    }
  }
  /* :275-319: the list of each site -- itself, then every later site within 0.5 A under some cell
   * translation, in site order (a site matched by several translations appears once: the repeats
   * the reference appends carry the same element and occupancy and never change a choice) */
  int st[3], fin[3];
  for (int k = 0; k < 3; k++) {
    st[k] = b->ncell[k] == 1 ? 0 : -2;
    fin[k] = b->ncell[k] == 1 ? 1 : 3;
  }
  size_t *off = (size_t *)malloc(((size_t)S + 1) * sizeof(size_t)), cap = 2 * (size_t)S + 16, L = 0;
  uint32_t *list = (uint32_t *)malloc(cap * sizeof(uint32_t));
  double *cum = (double *)malloc(cap * sizeof(double));
  for (uint32_t i = 0; i < S; i++) {
    off[i] = L;
    if (L + 1 > cap) cap *= 2, list = (uint32_t *)realloc(list, cap * 4), cum = (double *)realloc(cum, cap * 8);
    list[L] = i;
    cum[L] = b->occ[i / b->nsymm];
    L++;
    for (uint32_t j = i + 1; j < S; j++) {
      int hit = 0;
      for (int cx = st[0]; cx < fin[0] && !hit; cx++)
        for (int cy = st[1]; cy < fin[1] && !hit; cy++)
          for (int cz = st[2]; cz < fin[2] && !hit; cz++) {
            double d[3];
            for (int k = 0; k < 3; k++) {
              double ct = b->e[0][k] * (double)cx + b->e[1][k] * (double)cy + b->e[2][k] * (double)cz;
              d[k] = cell[3 * i + k] - cell[3 * j + k] + ct;
            }
            hit = d[0] * d[0] + d[1] * d[1] + d[2] * d[2] < 0.25;
          }
      if (!hit) continue;
      if (L + 1 > cap) cap *= 2, list = (uint32_t *)realloc(list, cap * 4), cum = (double *)realloc(cum, cap * 8);
      /* :305-306: add the occupancy only when the element differs from the previous entry's */
      cum[L] = type[j] != type[list[L - 1]] ? cum[L - 1] + b->occ[j / b->nsymm] : cum[L - 1];
      list[L] = j;
      L++;
    }
  }
  off[S] = L;
  double rmc[3] = {0, 0, 0};
  for (uint32_t c = 0; c < b->ncopy; c++)
    for (int k = 0; k < 3; k++) rmc[k] += b->r_copy[3 * c + k];
  for (int k = 0; k < 3; k++) rmc[k] /= (double)b->ncopy;
  unsigned char *claimed = (unsigned char *)malloc(S ? S : 1);
  for (uint32_t k = 0; k < b->nid; k++) n_all[k] = 0;
  uint64_t unit = 0;
  for (uint32_t c = 0; c < b->ncopy; c++)
    for (uint32_t cx = 0; cx < b->ncell[0]; cx++)
      for (uint32_t cy = 0; cy < b->ncell[1]; cy++)
        for (uint32_t cz = 0; cz < b->ncell[2]; cz++, unit++) {
          double ct[3];
          for (int k = 0; k < 3; k++) ct[k] = b->e[0][k] * (double)cx + b->e[1][k] * (double)cy + b->e[2][k] * (double)cz;
          memset(claimed, 0, S);
          for (uint32_t i = 0; i < S; i++) {
            if (claimed[i]) continue;
            for (size_t m = off[i]; m < off[i + 1]; m++) claimed[list[m]] = 1;
            double randval, unused;
            rng_draw(&g, i, unit, XO_P_OCC, &randval, &unused);
            size_t m = off[i];
            while (m < off[i + 1] && !(randval <= cum[m])) m++;
            if (m == off[i + 1]) continue;
            const uint32_t s = list[m], ia = s / b->nsymm, is = s % b->nsymm;
            double ra1[3] = {ra0[3 * s], ra0[3 * s + 1], ra0[3 * s + 2]};
            if (b->ro_mol) { /* :341-347, :358 */
              double u0, u1, u2, u3;
              rng_draw(&g, is, unit, XO_P_ROT_A, &u0, &u1);
              rng_draw(&g, is, unit, XO_P_ROT_B, &u2, &u3);
              double ex = 2.0 * XO_PI * u0, ey = XO_PI * u1, ez = 2.0 * XO_PI * u2;
              double cx_ = cos(ex), cy_ = cos(ey), cz_ = cos(ez), sx = sin(ex), sy = sin(ey), sz = sin(ez);
              double r0[3] = {cx_ * cy_ - sx * sy * cz_, -cx_ * sy - sx * cz_ * cy_, sx * sz};
              double r1[3] = {sx * cy_ + cx_ * sy * cz_, -sx * sy + cx_ * cy_ * cz_, -cx_ * sz};
              double r2[3] = {sz * sy, sz * cy_, cz_};
              double t[3] = {dot3(ra1, r0), dot3(ra1, r1), dot3(ra1, r2)};
              memcpy(ra1, t, sizeof t);
            }
            double rmd[3] = {0, 0, 0};
            if (b->dev_mol >= 1.e-7) rng_displacement(&g, is, unit, XO_P_MOL_ANG, XO_P_MOL_RAD, b->dev_mol, rmd);
            for (int k = 0; k < 3; k++) ra1[k] += b->r_symm[3 * is + k] + ct[k] + rmd[k]; /* :360 */
            double d[3];
            for (int k = 0; k < 3; k++) d[k] = ra1[k] - b->r_mean[k];
            if (b->cutoff && !(dot3(d, d) <= b->rcut * b->rcut)) continue; /* :361 */
            const double *cf = b->cf + 9 * c;
            double tr[3] = {dot3(d, cf), dot3(d, cf + 3), dot3(d, cf + 6)};
            for (int k = 0; k < 3; k++) ra1[k] = b->r_copy[3 * c + k] + tr[k];
            if (b->dev[ia] >= 1.e-7) { /* :364-371 */
              double dd[3];
              rng_displacement(&g, i, unit, XO_P_DISP_ANG, XO_P_DISP_RAD, b->dev[ia], dd);
              for (int k = 0; k < 3; k++) ra1[k] += dd[k];
            }
            if (b->cutoff_copies) { /* :372 */
              double e3[3];
              for (int k = 0; k < 3; k++) e3[k] = ra1[k] - rmc[k];
              if (!(dot3(e3, e3) <= b->rcut_copies * b->rcut_copies)) continue;
            }
            list_push(&out[b->id[type[s]]], ra1);
            n_all[type[s]]++;
          }
        }
  free(claimed);
  free(off);
  free(list);
  free(cum);
  free(ra0);
  free(cell);
  free(type);
}

double *xo_build_atoms(const xo_block *blocks, uint32_t nblocks, uint32_t nel, uint64_t seed, uint32_t *n_el,
                       uint32_t *n_all) {
  xo_list *out = (xo_list *)calloc(nel, sizeof(xo_list));
  uint32_t o_all = 0;
  for (uint32_t ib = 0; ib < nblocks; ib++) {
    uint32_t tmp[64];
    uint32_t *na = n_all ? n_all + o_all : tmp;
    if (blocks[ib].natom)
      build_block(&blocks[ib], ib, seed, out, na);
    else
      for (uint32_t k = 0; k < blocks[ib].nid; k++) na[k] = 0;
    o_all += blocks[ib].nid;
  }
  size_t tot = 0;
  for (uint32_t e = 0; e < nel; e++) tot += out[e].n;
  double *xyz = (double *)malloc(3 * (tot ? tot : 1) * sizeof(double));
  size_t o = 0;
  for (uint32_t e = 0; e < nel; e++) {
    n_el[e] = (uint32_t)out[e].n;
    if (out[e].n) memcpy(xyz + 3 * o, out[e].xyz, 3 * out[e].n * sizeof(double));
    o += out[e].n;
    free(out[e].xyz);
  }
  free(out);
  return xyz;
}

/* ---- rearrangement correction ---------------------------------------------------------------- */

void xo_rearrangement_int(double *I0, const double *q, uint32_t nq, const xo_rearr_block *blocks, uint32_t nblocks,
                          uint32_t nel, int source, const double *ff, const double *sl, int partial, int polar,
                          double lambda, uint32_t ntot) {
  (void)nel;
  long long N = (long long)(unsigned int)(ntot * ntot); /* SQR(Ntot) in unsigned int, :471 */
  uint32_t nint = partial ? (nblocks + 1) * nq : nq;
  double *I = (double *)calloc(nint, sizeof(double)), *Itemp = (double *)malloc(nq * sizeof(double));
#define XO_W(e, iq) (source == XO_XRAY ? ff[(size_t)(e) * nq + (iq)] : sl[e])
  for (uint32_t iB = 0; iB < nblocks; iB++) {
    const xo_rearr_block *b = &blocks[iB];
    uint32_t iqST = partial ? nq : 0; /* every block writes the first slot, :478-479 */
    if (!b->rearrangement) continue;
    unsigned int coeff = b->coeff;
    uint32_t ibegin = 0;
    for (uint32_t iEl = 0; iEl < b->nid; iEl++) {
      uint32_t jbegin = 0, id = b->id[iEl];
      for (uint32_t jEl = 0; jEl < b->nid; jEl++) {
        uint32_t jd = b->id[jEl];
        for (uint32_t iq = 0; iq < nq; iq++) Itemp[iq] = 0;
        for (uint32_t ia = ibegin; ia < ibegin + b->natom_el[iEl]; ia++) {
          const double *ri = b->r_atom + 3 * ia;
          double rmax2 = 0; /* Rmax2, :244-250 */
          for (uint32_t k = b->neighb_off[ia]; k < b->neighb_off[ia + 1]; k++) {
            const double *rn = b->neighb_r + 3 * k;
            double dx = ri[0] - rn[0], dy = ri[1] - rn[1], dz = ri[2] - rn[2];
            double d2 = dx * dx + dy * dy + dz * dz;
            rmax2 = rmax2 > d2 ? rmax2 : d2;
          }
          rmax2 = rmax2 + b->rcorr * b->rcorr;
          for (uint32_t ja = jbegin; ja < jbegin + b->natom_el[jEl]; ja++) {
            const double *rj = b->r_atom + 3 * ja;
            double dx = ri[0] - rj[0], dy = ri[1] - rj[1], dz = ri[2] - rj[2];
            double rij2 = dx * dx + dy * dy + dz * dz;
            if ((rij2 < rmax2) && (rij2 > 0.000001)) {
              N -= coeff;
              double rij = sqrt(rij2);
              for (uint32_t iq = 0; iq < nq; iq++) {
                double qrij = rij * q[iq];
                Itemp[iq] += sin(qrij) / (qrij + 0.00000001);
              }
            }
          }
        }
        for (uint32_t iq = 0; iq < nq; iq++) I[iqST + iq] -= (coeff * XO_W(id, iq) * XO_W(jd, iq)) * Itemp[iq];
        jbegin += b->natom_el[jEl];
      }
      for (uint32_t ia = ibegin; ia < ibegin + b->natom_el[iEl]; ia++) {
        const double *ri = b->r_atom + 3 * ia;
        for (uint32_t k = b->neighb_off[ia]; k < b->neighb_off[ia + 1]; k++) {
          const double *rn = b->neighb_r + 3 * k;
          uint32_t idN = b->neighb_id[k];
          double dx = ri[0] - rn[0], dy = ri[1] - rn[1], dz = ri[2] - rn[2];
          double rij = sqrt(dx * dx + dy * dy + dz * dz);
          N += coeff;
          for (uint32_t iq = 0; iq < nq; iq++) {
            double qrij = rij * q[iq];
            I[iqST + iq] += (coeff * XO_W(id, iq) * XO_W(idN, iq)) * sin(qrij) / (qrij + 0.00000001);
          }
        }
      }
      ibegin += b->natom_el[iEl];
    }
  }
#undef XO_W
  if (partial) {
    uint32_t iqST = nq;
    for (uint32_t iB = 0; iB < nblocks; iB++, iqST += nq) {
      uint32_t i0qST = nq * (1 + iB * (2 * nblocks - iB + 1) / 2);
      if (polar) polar_1d(I + iqST, q, lambda, nq);
      for (uint32_t iq = 0; iq < nq; iq++) {
        I[iq] += I[iqST + iq];
        I0[i0qST + iq] = (I0[i0qST + iq] * ntot + I[iqST + iq]) / sqrt((double)N);
      }
    }
  } else if (polar)
    polar_1d(I, q, lambda, nq);
  for (uint32_t iq = 0; iq < nq; iq++) I0[iq] = (I0[iq] * ntot + I[iq]) / sqrt((double)N);
  free(I);
  free(Itemp);
}
