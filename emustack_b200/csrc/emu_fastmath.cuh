// Reciprocals for the FP64 film recursion.
//
// A division in IEEE double costs a long dependent instruction sequence; the
// film kernel needs several per order and layer.  Here 1/a is computed by
// Newton-Raphson iteration for the reciprocal, x <- x (2 - a x), which
// doubles the number of correct bits per step, seeded with the
// single-precision reciprocal of a (about 23 correct bits): two steps give a
// result within a few ulps of 1/a in double.  Arguments whose magnitude is
// outside the single-precision normal range, and non-finite ones, take the
// IEEE division instead.
#pragma once
#include "emu_cplx.cuh"

namespace emu {

__device__ __forceinline__ double rcp_nr(double a) {
  const double aa = fabs(a);
  if (!(aa > 1e-36 && aa < 1e36)) return 1.0 / a;
  double x = (double)__frcp_rn((float)a);
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

// Principal square root (C99 csqrt branch rules) with the final quotient
// y / (2t) taken through rcp_nr.
__device__ __forceinline__ cd csqrt_nr(cd z) {
  if (z.x == 0.0 && z.y == 0.0) return cd{0.0, z.y};
  const double t = sqrt(0.5 * (fabs(z.x) + sqrt(fma(z.x, z.x, z.y * z.y))));
  const double h = 0.5 * rcp_nr(t);
  if (z.x >= 0.0) return cd{t, z.y * h};
  return cd{fabs(z.y) * h, copysign(t, z.y)};
}

}  // namespace emu
