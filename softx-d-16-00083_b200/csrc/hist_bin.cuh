// The reference's pair-distance bin, bit for bit.
//
// The reference bins (unsigned int)(rij / bin) with rij = sqrt((dx*dx + dy*dy) + dz*dz) evaluated in
// IEEE FP64 without FMA (vect3d::mag, typedefs.h:130, built by g++ -O3 for x86-64, which has no FMA):
// CalcFunctions.cpp:783-788.  ref_dist2 forms d2 with explicitly rounded FP64 operations in that
// order; ref_bin decides the bin from d2 with a cheap estimate that is exact whenever it is not within
// a proven margin of a bin edge, and with correctly rounded sqrt and divide otherwise.
#pragma once
#include <stdint.h>

namespace xns_hist {

// Float with the exponent and top 20 mantissa bits of d (d in [2^-126, 2^128)), built with integer
// operations only: the estimate needs no conversion-pipe instruction.
__device__ __forceinline__ float trunc_to_float(double d) {
  int hi = __double2hiint(d);
  return __int_as_float((hi - (896 << 20)) << 3);
}

__device__ __forceinline__ double float_to_double_exact(float f) {
  int b = __float_as_int(f);
  return __hiloint2double((b >> 3) + (896 << 20), b << 29);
}

// Reference bin index (unsigned)(fl(fl(sqrt(d2)) / bin)), or 0xffffffff when it is >= nhist.
//
// Estimate: f = d2 truncated to float (rel. err < 2^-20), y = rsqrtf(f) (max error 2 ulp, CUDA
// Programming Guide), so y = (1 + e)/sqrt(d2) with |e| < 0.75*2^-20.  One Newton step in FP64,
// r1 = r0 + (d2 - r0^2) * y/2 with r0 = d2*y, leaves |r1/sqrt(d2) - 1| < 2^-39.8, and
// t = r1 * fl(1/bin) is within t*2^-39.7 of the reference quotient Q = fl(fl(sqrt(d2))/bin)
// (itself within 2^-52 of sqrt(d2)/bin).  With t < nhist, any |t - round(t)| >= margin =
// nhist*2^-37 proves floor(Q) = floor(t); otherwise the exact IEEE operations decide.
__device__ __forceinline__ uint32_t ref_bin(double d2, double bin, double inv_bin, double margin, uint32_t nhist) {
  const double MAGIC = 6755399441055744.0;  // 1.5 * 2^52: adding it rounds to an integer in the low word
  int hi = __double2hiint(d2);
  if (hi >= (897 << 20) && hi < (1151 << 20)) {
    float y = rsqrtf(trunc_to_float(d2));
    double yd = float_to_double_exact(y);
    double r0 = __dmul_rn(d2, yd);
    double res = __fma_rn(-r0, r0, d2);
    double r1 = __fma_rn(res, 0.5 * yd, r0);
    double t = __dmul_rn(r1, inv_bin);
    if (t < (double)nhist - 1.0) {
      double u = __dadd_rn(t, MAGIC);
      double v = __dsub_rn(u, MAGIC);
      double d = __dsub_rn(t, v);
      if (fabs(d) >= margin) return (uint32_t)__double2loint(u) - (d < 0.0 ? 1u : 0u);
    }
  }
  double q = __ddiv_rn(__dsqrt_rn(d2), bin);
  if (!(q < (double)nhist)) return 0xffffffffu;
  return (uint32_t)q;
}

// The estimate of ref_bin without branches: k is valid when the return value is true.  Callers run
// several of these side by side (independent FP64 chains) and send the rare false ones to ref_bin.
__device__ __forceinline__ bool ref_bin_fast(double d2, double inv_bin, double margin, double nhist_m1, uint32_t *k) {
  const double MAGIC = 6755399441055744.0;
  const int hi = __double2hiint(d2);
  const bool in_range = (unsigned)(hi - (897 << 20)) < (unsigned)((1151 - 897) << 20);
  // rsqrt.approx (what rsqrtf compiles to; 2 ulp): the flush-to-zero form is one MUFU instruction, and
  // in_range keeps its argument a normal float
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(trunc_to_float(d2)));
  const double yd = float_to_double_exact(y);
  const double r0 = __dmul_rn(d2, yd);
  const double res = __fma_rn(-r0, r0, d2);
  const double t = __dmul_rn(__fma_rn(res, 0.5 * yd, r0), inv_bin);
  const double u = __dadd_rn(t, MAGIC);
  const double d = __dsub_rn(t, __dsub_rn(u, MAGIC));
  *k = (uint32_t)__double2loint(u) - (d < 0.0 ? 1u : 0u);
  return in_range && t < nhist_m1 && fabs(d) >= margin;
}

__device__ __forceinline__ double ref_dist2(double xi, double yi, double zi, double xj, double yj, double zj) {
  double dx = __dsub_rn(xi, xj), dy = __dsub_rn(yi, yj), dz = __dsub_rn(zi, zj);
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

}  // namespace xns_hist
