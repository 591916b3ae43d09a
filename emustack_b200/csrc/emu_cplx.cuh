// Complex double arithmetic for the GSM kernels.
//
// The operations follow the same formulas numpy uses for complex128 so that
// results stay within a few ulps of the reference:
//   * division: R. L. Smith, "Algorithm 116: Complex division", CACM 5(8), 1962;
//   * square root: principal branch with C99 csqrt semantics (branch cut on
//     the negative real axis, the sign of a zero imaginary part selects the
//     side), evaluated as t = sqrt((|x| + |z|)/2) (W. Kahan, "Branch cuts for
//     complex elementary functions", 1987);
//   * exponential: exp(x) * (cos y, sin y).
#pragma once
#include <cuda_runtime.h>
#include <math.h>

struct cd {
  double x, y;
};

__host__ __device__ __forceinline__ cd mkc(double x, double y) { return cd{x, y}; }
__host__ __device__ __forceinline__ cd cadd(cd a, cd b) { return cd{a.x + b.x, a.y + b.y}; }
__host__ __device__ __forceinline__ cd csub(cd a, cd b) { return cd{a.x - b.x, a.y - b.y}; }
__host__ __device__ __forceinline__ cd cneg(cd a) { return cd{-a.x, -a.y}; }
__host__ __device__ __forceinline__ cd cconj(cd a) { return cd{a.x, -a.y}; }
__host__ __device__ __forceinline__ cd cscale(cd a, double s) { return cd{a.x * s, a.y * s}; }
// Products and squared magnitudes with their roundings written out (one
// rounded product, one fused multiply-add), so that every kernel inlining
// them rounds alike whatever contraction the compiler would choose.
__host__ __device__ __forceinline__ double rmul(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
__host__ __device__ __forceinline__ cd cmul(cd a, cd b) {
  return cd{fma(a.x, b.x, -rmul(a.y, b.y)), fma(a.x, b.y, rmul(a.y, b.x))};
}
__host__ __device__ __forceinline__ double cabs2(cd a) { return fma(a.x, a.x, rmul(a.y, a.y)); }
__host__ __device__ __forceinline__ double cabsd(cd a) { return hypot(a.x, a.y); }
__host__ __device__ __forceinline__ bool cis_zero(cd a) { return a.x == 0.0 && a.y == 0.0; }

// Smith's algorithm.
__host__ __device__ __forceinline__ cd cdiv(cd a, cd b) {
  if (fabs(b.x) >= fabs(b.y)) {
    if (b.x == 0.0 && b.y == 0.0) {
      return cd{a.x / fabs(b.x), a.y / fabs(b.y)};  // IEEE inf/nan like numpy
    }
    double r = b.y / b.x;
    double den = b.x + b.y * r;
    return cd{(a.x + a.y * r) / den, (a.y - a.x * r) / den};
  } else {
    double r = b.x / b.y;
    double den = b.x * r + b.y;
    return cd{(a.x * r + a.y) / den, (a.y * r - a.x) / den};
  }
}

// 1 / b for a real numerator.
__host__ __device__ __forceinline__ cd crecip(cd b) { return cdiv(cd{1.0, 0.0}, b); }

// Principal square root, C99 csqrt semantics for finite arguments.
__host__ __device__ __forceinline__ cd csqrt_p(cd z) {
  if (z.x == 0.0 && z.y == 0.0) return cd{0.0, z.y};
  double t = sqrt(0.5 * (fabs(z.x) + hypot(z.x, z.y)));
  if (z.x >= 0.0) return cd{t, z.y / (2.0 * t)};
  return cd{fabs(z.y) / (2.0 * t), copysign(t, z.y)};
}

// exp(z)
__device__ __forceinline__ cd cexp_d(cd z) {
  double s, c;
  sincos(z.y, &s, &c);
  double e = exp(z.x);
  return cd{e * c, e * s};
}

// exp(i * z * h) as numpy evaluates np.exp(1j * z * h): (1j*z) = (-z.y, z.x),
// then times the real h.
__device__ __forceinline__ cd cexp_ikh(cd z, double h) {
  return cexp_d(cd{-z.y * h, z.x * h});
}
