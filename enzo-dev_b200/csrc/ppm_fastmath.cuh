// ppm_fastmath.cuh -- reciprocal, quotient, square root and reciprocal square root for
// the tolerance-mode build.
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
//   per step (20 -> 40 -> 80), two steps;
// - reciprocal square root: with e = 1 - x*y0^2, the cubic truncation of the series
//   (1 - e)^(-1/2) = 1 + e/2 + 3e^2/8 + ... (relative error about (5/16) e^3).
//
// Measured on a B200 against CUDA's IEEE division and sqrt over 3.2e9 random operands
// (exponents over +-60, +-1000 and near 1): at most 1 ulp apart for the reciprocal,
// the quotient and the square root, 1.22 ulp for the reciprocal square root.
//
// No branches: the special arguments are picked out on the integer pipe from the
// exponent bits and their results selected.  Zeros, infinities and NaN give the IEEE
// results; subnormal arguments count as zero and results that would be subnormal flush
// to zero (the hardware approximations' ftz).  Branch-free code also keeps the results
// independent of where the compiler places them: with a branch around the IEEE
// fallback, the multiply-adds fused around these calls differed between kernel
// instantiations, and a level solved in one batch stopped matching the same grids
// solved one at a time.  In the exact build (PPM_FAST_ALGEBRA 0) they are the IEEE
// operations themselves.
#pragma once

#ifndef PPM_FAST_ALGEBRA
#define PPM_FAST_ALGEBRA 0
#endif
#ifndef PPM_FAST_DIVSQRT
#define PPM_FAST_DIVSQRT PPM_FAST_ALGEBRA
#endif

namespace ppm {

// biased exponent of x
__device__ __forceinline__ unsigned fm_exponent(double x) {
  return ((unsigned)__double2hiint(x) >> 20) & 0x7FFu;
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
  const double y0 = fm_rcp_approx(x);
  const double e = fma(-x, y0, 1.0);
  const double r = fma(y0, fma(e, e, e), y0);
  // |x| in [2^-1022, 2^1021): x and 1/x normal; otherwise the approximation itself is
  // exact (+-0 -> +-inf, +-inf -> +-0, NaN) or flushed (subnormal x, subnormal 1/x)
  return fm_exponent(x) - 1u <= 2042u ? r : y0;
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

// 1/sqrt(x): with e = 1 - x*y0^2, (1 - e)^(-1/2) = 1 + e/2 + 3e^2/8 + ...; the cubic
// truncation leaves a relative error of about (5/16) e^3 (2^-61)
__device__ __forceinline__ double qrsqrt(double x) {
#if PPM_FAST_DIVSQRT
  const double y0 = fm_rsqrt_approx(x);
  const double e = fma(-x * y0, y0, 1.0);
  const double y1 = fma(y0, e * fma(0.375, e, 0.5), y0);
  // normal x: y1 (NaN for x < 0); +-0 -> +-inf, +inf -> 0, NaN: the approximation itself
  return fm_exponent(x) - 1u <= 2045u ? y1 : y0;
#else
  return 1.0 / sqrt(x);
#endif
}

// sqrt(x)
__device__ __forceinline__ double qsqrt(double x) {
#if PPM_FAST_DIVSQRT
  const double y0 = fm_rsqrt_approx(x);  // NaN for x < 0, which the iteration keeps
  double g = x * y0, h = 0.5 * y0;
  double r = fma(-g, h, 0.5);
  g = fma(g, r, g);
  h = fma(h, r, h);
  r = fma(-g, h, 0.5);
  const double s = fma(g, r, g);
  const unsigned ex = fm_exponent(x);
  const int hi = __double2hiint(x);
  // exponent 0: +-0 (and subnormals, flushed) -> +-0; exponent 2047: +inf -> +inf,
  // -inf -> NaN, NaN -> NaN
  const double special = ex == 0u ? __hiloint2double(hi & (int)0x80000000, 0)
                                  : (hi < 0 ? __longlong_as_double(0x7FF8000000000000ll) : x);
  return ex - 1u <= 2045u ? s : special;
#else
  return sqrt(x);
#endif
}

}  // namespace ppm
