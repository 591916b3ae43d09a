// Reciprocals and square roots for the FP64 film recursion.
//
// A division in IEEE double costs a long dependent instruction sequence; the
// film kernel needs several per order and layer.  Here 1/a is computed by
// Newton-Raphson iteration for the reciprocal, x <- x (2 - a x), which
// doubles the number of correct bits per step, seeded with the hardware's
// approximate double reciprocal (rcp.approx.ftz.f64): two steps give a result
// within a few ulps of 1/a (the film outputs agree with those of IEEE
// divisions to 1e-15 absolute).  Arguments whose magnitude is outside
// [1e-300, 1e300], and non-finite ones, take the IEEE division instead.
#pragma once
#include "emu_cplx.cuh"

namespace emu {

__device__ __forceinline__ double rcp_nr(double a) {
  const double aa = fabs(a);
  if (!(aa > 1e-300 && aa < 1e300)) return 1.0 / a;
  double x;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(x) : "d"(a));
  double e = fma(-a, x, 1.0);
  x = fma(x, e, x);
  e = fma(-a, x, 1.0);
  x = fma(x, e, x);
  return x;
}

// 1 / z = conj(z) / |z|^2
__device__ __forceinline__ cd crcp_nr(cd z) {
  const double r = rcp_nr(fma(z.x, z.x, z.y * z.y));
  return cd{z.x * r, -z.y * r};
}

// 1/sqrt(a) for a normal positive a: Newton-Raphson for the reciprocal
// square root, y <- y (3/2 - a y^2 / 2), seeded with the hardware's
// approximate double reciprocal square root (rsqrt.approx.ftz.f64); two
// steps, as for rcp_nr.
__device__ __forceinline__ double rsqrt_nr(double a) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
  const double ha = 0.5 * a;
  double e = fma(-ha * y, y, 0.5);
  y = fma(y, e, y);
  e = fma(-ha * y, y, 0.5);
  y = fma(y, e, y);
  return y;
}

// Principal square root for k_z (C99 csqrt branch rules, Kahan's form
// t = sqrt((|x| + |z|)/2)) from two reciprocal square roots: |z| = q / sqrt(q)
// with q = |z|^2, t = s / sqrt(s) and 1/(2t) = 1/(2 sqrt(s)) with
// s = (|x| + |z|)/2.  Where |z|^2 would leave the normal range (and for zero
// or non-finite z) it takes the IEEE form csqrt_p.  Both give exact zeros
// and exactly real or exactly imaginary results for the same arguments.
__device__ __forceinline__ cd csqrt_k(cd z) {
  const double ax = fabs(z.x), ay = fabs(z.y);
  const double m = fmax(ax, ay);
  if (!(m > 1e-150 && m < 1e150)) return csqrt_p(z);
  const double q = fma(z.x, z.x, z.y * z.y);
  const double h = q * rsqrt_nr(q);
  const double sh = 0.5 * (ax + h);
  const double r = rsqrt_nr(sh);
  const double t = sh * r;
  const double hr = 0.5 * r;
  if (z.x >= 0.0) return cd{t, z.y * hr};
  return cd{ay * hr, copysign(t, z.y)};
}

// csqrt_p(z).y == 0 (the order propagates) decided from z itself: the
// principal root is real exactly when z is real and not negative.
__device__ __forceinline__ bool sqrt_is_real(cd z) { return z.y == 0.0 && z.x >= 0.0; }

}  // namespace emu
