// Accurate sine and cosine of an FP64 phase on the FMA pipes.
//
// The MUFU approximations (__sinf / __sincosf, max abs error ~2^-21.4) have an error that varies
// smoothly with the argument.  Pair distances in a crystal come in shells whose phases q*r differ by
// far less than that error's period, so the MUFU error adds up coherently over a shell and limits
// I(q) to ~1e-4 relative at its minima.  xns_sincos instead reduces the phase to one quadrant in FP64
// (x = n*pi/2 + y, |y| <= pi/4 + tiny) and evaluates the Taylor series of sin and cos in FP32:
//   sin y = y - y^3/3! + y^5/5! - y^7/7! + y^9/9!        (truncation < 2e-9 on |y| <= pi/4)
//   cos y = 1 - y^2/2! + y^4/4! - ... - y^10/10!        (truncation < 2e-10)
// so the result carries FP32 rounding only (a few 1e-8, uncorrelated between arguments).  Valid for
// |x| < 2^50.
#pragma once

namespace xns_math {

__device__ __forceinline__ void sincos_quadrant(float y, int n, float *s, float *c) {
  const float y2 = y * y;
  float sp = fmaf(y2, 2.75573192e-6f, -1.98412698e-4f);  // 1/9!, -1/7!
  sp = fmaf(y2, sp, 8.33333333e-3f);                      // 1/5!
  sp = fmaf(y2, sp, -1.66666667e-1f);                     // -1/3!
  sp = fmaf(y2 * y, sp, y);
  float cp = fmaf(y2, -2.75573192e-7f, 2.48015873e-5f);   // -1/10!, 1/8!
  cp = fmaf(y2, cp, -1.38888889e-3f);                     // -1/6!
  cp = fmaf(y2, cp, 4.16666667e-2f);                      // 1/4!
  cp = fmaf(y2, cp, -0.5f);                               // -1/2!
  cp = fmaf(y2, cp, 1.0f);
  // quadrant n mod 4: (sin, cos) = (sp, cp), (cp, -sp), (-sp, -cp), (-cp, sp)
  const float a = (n & 1) ? cp : sp, b = (n & 1) ? sp : cp;
  *s = (n & 2) ? -a : a;
  *c = ((n + 1) & 2) ? -b : b;
}

// sin and cos of x (radians, FP64).
__device__ __forceinline__ void xns_sincos(double x, float *s, float *c) {
  const double MAGIC = 6755399441055744.0;  // 1.5 * 2^52: rounds to an integer kept in the low word
  const double TWO_OVER_PI = 0.63661977236758134308;
  const double PIO2_HI = 1.5707963267948966192;   // pi/2 rounded to FP64
  const double PIO2_LO = 6.123233995736766036e-17; // pi/2 - PIO2_HI
  const double t = __fma_rn(x, TWO_OVER_PI, MAGIC);
  const int n = __double2loint(t);
  const double nd = t - MAGIC;
  const double y = __fma_rn(-nd, PIO2_LO, __fma_rn(-nd, PIO2_HI, x));
  sincos_quadrant((float)y, n, s, c);
}

// sin and cos of x (radians) in FP64: the same quadrant reduction, then the Taylor series in FP64,
//   sin y = y - y^3/3! + ... - y^11/11!   (truncation < 1e-11 on |y| <= pi/4)
//   cos y = 1 - y^2/2! + ... - y^10/10!   (truncation < 2e-10)
// for seeds that must round to FP32 correctly: the FP32 series above leaves one or two FP32 ulps,
// which at the deep minima of a Debye pattern (a sum that cancels to 1e-5 of its terms) is visible.
// Runs on the FP64 pipe, beside the FP32 work of the sinc engine.  Valid for |x| < 2^50.
__device__ __forceinline__ void xns_sincos64(double x, double *s, double *c) {
  const double MAGIC = 6755399441055744.0;
  const double TWO_OVER_PI = 0.63661977236758134308;
  const double PIO2_HI = 1.5707963267948966192;
  const double PIO2_LO = 6.123233995736766036e-17;
  const double t = __fma_rn(x, TWO_OVER_PI, MAGIC);
  const int n = __double2loint(t);
  const double nd = t - MAGIC;
  const double y = __fma_rn(-nd, PIO2_LO, __fma_rn(-nd, PIO2_HI, x));
  const double y2 = y * y;
  double sp = __fma_rn(y2, -1.0 / 39916800.0, 1.0 / 362880.0);  // -1/11!, 1/9!
  sp = __fma_rn(y2, sp, -1.0 / 5040.0);                          // -1/7!
  sp = __fma_rn(y2, sp, 1.0 / 120.0);                            // 1/5!
  sp = __fma_rn(y2, sp, -1.0 / 6.0);                             // -1/3!
  sp = __fma_rn(y2 * y, sp, y);
  double cp = __fma_rn(y2, -1.0 / 3628800.0, 1.0 / 40320.0);    // -1/10!, 1/8!
  cp = __fma_rn(y2, cp, -1.0 / 720.0);                           // -1/6!
  cp = __fma_rn(y2, cp, 1.0 / 24.0);                             // 1/4!
  cp = __fma_rn(y2, cp, -0.5);                                   // -1/2!
  cp = __fma_rn(y2, cp, 1.0);
  const double a = (n & 1) ? cp : sp, b = (n & 1) ? sp : cp;
  *s = (n & 2) ? -a : a;
  *c = ((n + 1) & 2) ? -b : b;
}

__device__ __forceinline__ float xns_sin(double x) {
  float s, c;
  xns_sincos(x, &s, &c);
  return s;
}

// sin and cos of x in FP64 to about one ulp for |x| < 2^20: the same quadrant reduction, then the
// Taylor series of sin y to y^15 and of cos y to y^16 (truncation below 5e-17 on |y| <= pi/4), for
// values that enter FP64 sums (the angle-split transforms).
__device__ __forceinline__ void xns_sincos64_acc(double x, double *s, double *c) {
  const double MAGIC = 6755399441055744.0;  // 1.5 * 2^52: rounds to an integer kept in the low word
  const double TWO_OVER_PI = 0.63661977236758134308;
  const double PIO2_HI = 1.5707963267948966192;
  const double PIO2_LO = 6.123233995736766036e-17;
  const double t = __fma_rn(x, TWO_OVER_PI, MAGIC);
  const int n = __double2loint(t);
  const double nd = t - MAGIC;
  const double y = __fma_rn(-nd, PIO2_LO, __fma_rn(-nd, PIO2_HI, x));
  const double y2 = y * y;
  double sp = __fma_rn(y2, -1.0 / 1307674368000.0, 1.0 / 6227020800.0);  // -1/15!, 1/13!
  sp = __fma_rn(y2, sp, -1.0 / 39916800.0);                               // -1/11!
  sp = __fma_rn(y2, sp, 1.0 / 362880.0);                                  // 1/9!
  sp = __fma_rn(y2, sp, -1.0 / 5040.0);                                   // -1/7!
  sp = __fma_rn(y2, sp, 1.0 / 120.0);                                     // 1/5!
  sp = __fma_rn(y2, sp, -1.0 / 6.0);                                      // -1/3!
  sp = __fma_rn(y2 * y, sp, y);
  double cp = __fma_rn(y2, 1.0 / 20922789888000.0, -1.0 / 87178291200.0);  // 1/16!, -1/14!
  cp = __fma_rn(y2, cp, 1.0 / 479001600.0);                                  // 1/12!
  cp = __fma_rn(y2, cp, -1.0 / 3628800.0);                                   // -1/10!
  cp = __fma_rn(y2, cp, 1.0 / 40320.0);                                      // 1/8!
  cp = __fma_rn(y2, cp, -1.0 / 720.0);                                       // -1/6!
  cp = __fma_rn(y2, cp, 1.0 / 24.0);                                         // 1/4!
  cp = __fma_rn(y2, cp, -0.5);                                               // -1/2!
  cp = __fma_rn(y2, cp, 1.0);
  const double a = (n & 1) ? cp : sp, b = (n & 1) ? sp : cp;
  *s = (n & 2) ? -a : a;
  *c = ((n + 1) & 2) ? -b : b;
}

}  // namespace xns_math
