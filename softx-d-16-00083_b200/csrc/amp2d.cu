// 2D scattering pattern on the reference's polar (q, phi) mesh (replaces calcInt2D,
// CalcFunctions.cpp:969-1091, and calcInt2DKernelXray/Neutron, CalcFunctionsCUDA.cu:567-650).
//
// For every orientation of the Euler mesh and every (q_i, phi_k):
//   qv = q_i (c cos phi, c sin phi, -s),  s = q_i lambda / 4pi,  c = 1 - s^2  (as the reference, :999-1002)
//   A  = sum_e w_e(q_i) sum_{j in e} exp(i (R^T qv) . r_j),   I2D += |A|^2
// then I2D *= 1/(Ntot N_orient), the polarisation factor, and I(q) = mean over phi (:1066-1076).
//
// One thread per mesh point; atoms are staged through shared memory in tiles shared by the CTA.
// The phase (R^T qv).r is formed and reduced in FP64 (it reaches ~10^3 rad for 10^6-atom
// crystallites, where an FP32 phase would carry ~1e-4 rad of error) and its sine and cosine come from
// the accurate polynomial of xmath.cuh (on a lattice the MUFU approximation's error adds coherently).
// Tile sums run in FP32 (<= 256 terms) and are added to FP64 amplitude totals (compensated block
// accumulation).
#include <math.h>
#include <string.h>

#include <algorithm>

#include "xmath.cuh"
#include "xns_internal.cuh"

namespace {

constexpr int A2_THREADS = 256;
constexpr int A2_TILE = 256;

__global__ void __launch_bounds__(A2_THREADS) amp2d_polar_kernel(
    const double *__restrict__ X, const double *__restrict__ Y, const double *__restrict__ Z,
    const uint32_t *__restrict__ off_el, uint32_t nel, const double *__restrict__ q, uint32_t nq, uint32_t nfi,
    const double *__restrict__ rot /* norient x 9, row-major R */, uint32_t norient, double lambda,
    const double *__restrict__ w /* nel x nq */, double norm, int polar, double *__restrict__ I2D) {
  __shared__ double sx[A2_TILE], sy[A2_TILE], sz[A2_TILE];
  const uint32_t pt = blockIdx.x * A2_THREADS + threadIdx.x;
  const bool valid = pt < nq * nfi;
  const uint32_t iq = valid ? pt / nfi : 0, ifi = valid ? pt % nfi : 0;
  const double qi = q[iq];
  const double st = qi * (lambda * 0.25 / XNS_PI), ct = 1. - st * st;
  const double dfi = 2. * XNS_PI / nfi;
  const double v0 = ct * cos(ifi * dfi) * qi, v1 = ct * sin(ifi * dfi) * qi, v2 = -st * qi;
  double inten = 0;
  for (uint32_t o = 0; o < norient; o++) {
    const double *m = rot + 9 * o;
    // R^T qv (CS rows are the columns of R, :1020-1022)
    const double w0 = v0 * m[0] + v1 * m[3] + v2 * m[6];
    const double w1 = v0 * m[1] + v1 * m[4] + v2 * m[7];
    const double w2 = v0 * m[2] + v1 * m[5] + v2 * m[8];
    double Ar = 0, Ai = 0;
    for (uint32_t e = 0; e < nel; e++) {
      double er = 0, ei = 0;
      for (uint32_t t0 = off_el[e]; t0 < off_el[e + 1]; t0 += A2_TILE) {
        const uint32_t n = min((uint32_t)A2_TILE, off_el[e + 1] - t0);
        __syncthreads();
        for (uint32_t j = threadIdx.x; j < n; j += A2_THREADS) {
          sx[j] = X[t0 + j];
          sy[j] = Y[t0 + j];
          sz[j] = Z[t0 + j];
        }
        __syncthreads();
        if (valid) {
          float tr = 0.f, ti = 0.f;
          for (uint32_t j = 0; j < n; j++) {
            float s, c;
            xns_math::xns_sincos(__fma_rn(w2, sz[j], __fma_rn(w1, sy[j], w0 * sx[j])), &s, &c);
            tr += c;
            ti += s;
          }
          er += tr;
          ei += ti;
        }
      }
      const double we = w[(size_t)e * nq + iq];
      Ar += we * er;
      Ai += we * ei;
    }
    inten += Ar * Ar + Ai * Ai;
  }
  if (!valid) return;
  double fac = norm;
  if (polar) {  // PolarFactor2D, CalcFunctions.cpp:451-459
    double s = qi * (lambda * 0.25 / XNS_PI), c2 = 1. - 2. * s * s;
    inten *= norm;
    fac = 0.5 * (1. + c2 * c2);
  }
  I2D[pt] = inten * fac;
}

// I(q) = (sum over phi of I2D) / Nfi, summed in the reference's order (:1072-1075)
__global__ void phi_mean_kernel(const double *__restrict__ I2D, uint32_t nq, uint32_t nfi, double *__restrict__ I) {
  const uint32_t iq = blockIdx.x * blockDim.x + threadIdx.x;
  if (iq >= nq) return;
  double s = 0;
  for (uint32_t k = 0; k < nfi; k++) s += I2D[(size_t)iq * nfi + k];
  I[iq] = s / nfi;
}

void rot_axis(int axis, double a, double m[9]) {
  double c = cos(a), s = sin(a);
  memset(m, 0, 9 * sizeof(double));
  if (axis == 0) { m[0] = 1; m[4] = c; m[5] = -s; m[7] = s; m[8] = c; }
  if (axis == 1) { m[4] = 1; m[0] = c; m[2] = s; m[6] = -s; m[8] = c; }
  if (axis == 2) { m[8] = 1; m[0] = c; m[1] = -s; m[3] = s; m[4] = c; }
}

void mat_mul(const double a[9], const double b[9], double out[9]) {
  double t[9];
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) t[3 * r + c] = a[3 * r] * b[c] + a[3 * r + 1] * b[3 + c] + a[3 * r + 2] * b[6 + c];
  memcpy(out, t, sizeof(t));
}

}  // namespace

// calcRotMatrix (CalcFunctions.cpp:46-115): convention "UVW" (typedefs.h:59-70) is the intrinsic
// product R_U(alpha) R_V(beta) R_W(gamma).
void xns_rot_matrix(const double euler[3], uint32_t convention, double m[9]) {
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

extern "C" int xns_calc_int_2d(xns_ctx *ctx, const double *const *xyz_el, const uint32_t *n_el, uint32_t nel, const double *q,
                               uint32_t nq, uint32_t nfi, const double *euler_min, const double *euler_max,
                               const uint32_t *euler_n, uint32_t convention, double lambda, int source,
                               const double *const *ff, const double *sl, int polar, double *I2D, double *I) {
  if (!ctx) return XNS_ERR_ARG;
  if (!q || !I2D || !I || nq == 0 || nfi == 0 || !euler_min || !euler_max || !euler_n || convention > 11)
    return xns_fail(ctx, XNS_ERR_ARG, "2D: null pointer, zero mesh size or bad Euler convention");
  if ((uint64_t)nq * nfi >= (1ull << 32)) return xns_fail(ctx, XNS_ERR_ARG, "2D: mesh too large");
  const uint64_t norient = (uint64_t)euler_n[0] * euler_n[1] * euler_n[2];
  if (norient == 0 || norient > (1u << 24)) return xns_fail(ctx, XNS_ERR_ARG, "2D: bad Euler mesh size");
  int st;
  DevCoords dc;
  if ((st = xns_upload_coords(ctx, xyz_el, n_el, nel, &dc))) return st;
  if (dc.ntot == 0) return xns_fail(ctx, XNS_ERR_ARG, "2D: no atoms");
  double *d_w;
  if ((st = xns_upload_weights(ctx, nel, nq, source, ff, sl, &d_w))) return st;
  // rotation matrices of the Euler mesh mid-points (:1007-1019), q mesh and element offsets
  double d[3];
  for (int k = 0; k < 3; k++) d[k] = euler_n[k] < 2 ? 0 : (euler_max[k] - euler_min[k]) / euler_n[k];
  const size_t rot_bytes = sizeof(double) * 9 * norient, q_bytes = sizeof(double) * nq, off_bytes = sizeof(uint32_t) * (nel + 1);
  const size_t aux_bytes = rot_bytes + q_bytes + off_bytes;
  void *aux, *h;
  if ((st = xns_scratch(ctx, SLOT_AUX, aux_bytes, &aux))) return st;
  if ((st = xns_pinned(ctx, aux_bytes, &h))) return st;
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  double *hr = (double *)h;
  size_t o = 0;
  for (uint32_t ia = 0; ia < euler_n[0]; ia++)
    for (uint32_t ib = 0; ib < euler_n[1]; ib++)
      for (uint32_t ig = 0; ig < euler_n[2]; ig++, o++) {
        double eul[3] = {euler_min[0] + (ia + 0.5) * d[0], euler_min[1] + (ib + 0.5) * d[1], euler_min[2] + (ig + 0.5) * d[2]};
        xns_rot_matrix(eul, convention, hr + 9 * o);
      }
  memcpy((char *)h + rot_bytes, q, q_bytes);
  uint32_t *hoff = (uint32_t *)((char *)h + rot_bytes + q_bytes);
  for (uint32_t e = 0; e < nel; e++) hoff[e] = dc.off_el[e];
  hoff[nel] = dc.ntot;
  XNS_CUDA(ctx, cudaMemcpyAsync(aux, h, aux_bytes, cudaMemcpyHostToDevice, ctx->stream));
  const double *d_rot = (const double *)aux, *d_q = (const double *)((char *)aux + rot_bytes);
  const uint32_t *d_off = (const uint32_t *)((char *)aux + rot_bytes + q_bytes);
  void *d_I2D, *d_I;
  if ((st = xns_scratch(ctx, SLOT_OUT, sizeof(double) * (size_t)nq * nfi, &d_I2D))) return st;
  if ((st = xns_scratch(ctx, SLOT_OUT2, sizeof(double) * nq, &d_I))) return st;
  const double norm = 1. / ((double)dc.ntot * euler_n[0] * euler_n[1] * euler_n[2]);
  if ((st = xns_timer_start(ctx))) return st;
  if ((st = xns_stage_begin(ctx, STAGE_2D))) return st;
  const uint32_t npts = nq * nfi;
  amp2d_polar_kernel<<<(npts + A2_THREADS - 1) / A2_THREADS, A2_THREADS, 0, ctx->stream>>>(
      dc.x, dc.y, dc.z, d_off, nel, d_q, nq, nfi, d_rot, (uint32_t)norient, lambda, d_w, norm, polar, (double *)d_I2D);
  XNS_LAUNCHED(ctx);
  phi_mean_kernel<<<(nq + 127) / 128, 128, 0, ctx->stream>>>((const double *)d_I2D, nq, nfi, (double *)d_I);
  XNS_LAUNCHED(ctx);
  if ((st = xns_stage_end(ctx, STAGE_2D))) return st;
  if ((st = xns_timer_stop(ctx))) return st;
  XNS_CUDA(ctx, cudaMemcpyAsync(I2D, d_I2D, sizeof(double) * (size_t)nq * nfi, cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaMemcpyAsync(I, d_I, sizeof(double) * nq, cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XNS_OK;
}
