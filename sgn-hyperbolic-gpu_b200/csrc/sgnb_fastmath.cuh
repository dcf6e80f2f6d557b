// sgnb_fastmath.cuh -- the fast arithmetic mode's reciprocal and square root.
//
// Both refine a hardware estimate by Newton-Raphson iterations (the methods are named
// below); the exact mode never uses them. Tested against the device's IEEE results in ulps
// (tests/test_fast_math_gpu.py through sgnb_fast_math).
#pragma once

namespace sgnb {
namespace dev {

// Reciprocal for the fast mode: the hardware estimate (PTX rcp.approx.ftz.f64) refined by
// two Newton-Raphson steps r <- r + r (1 - x r), each of which doubles the number of
// correct bits. For normal x (the positive depths and error scales it is used on); the
// GPU tests compare it with IEEE 1/x in ulps through sgnb_fast_math.
__device__ __forceinline__ double fast_rcp(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  double e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  return r;
}

// Square root for the fast mode, by Newton-Raphson on the reciprocal square root: the
// hardware estimate y of 1/sqrt(x) (PTX rsqrt.approx.ftz.f64), two steps
// y <- y (3/2 - (x/2) y^2), then s = x y and one Newton (Heron) step on s^2 = x written
// with the residual, s <- s + (y/2) (x - s^2). Normal finite x only; zero, subnormal,
// infinite, negative and NaN arguments take the IEEE square root. Tested against IEEE
// sqrt in ulps through sgnb_fast_math.
__device__ __forceinline__ double fast_sqrt(double x) {
  if (!(x >= 2.2250738585072014e-308 && x <= 1.7976931348623157e308)) return sqrt(x);
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double hx = 0.5 * x;
  y = y * fma(-hx * y, y, 1.5);
  y = y * fma(-hx * y, y, 1.5);
  const double s = x * y;
  return fma(0.5 * y, fma(-s, s, x), s);
}

}  // namespace dev
}  // namespace sgnb
