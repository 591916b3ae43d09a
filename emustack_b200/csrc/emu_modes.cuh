// Analytic film modes shared by the film kernels: plane-wave k_z, impedances,
// Fresnel interfaces and shear phases, in the reference's operation order
// (backend/mode_calcs.py:116-218, 451-477, 80-87).
#pragma once
#include "emu_cplx.cuh"

namespace emu {

constexpr double kPi = 3.141592653589793;

// k^2 - alpha^2 - beta^2 in numpy's evaluation order, no contraction.
__device__ __forceinline__ cd kz_arg(cd k, double alpha, double beta) {
  double re = __dsub_rn(__dmul_rn(k.x, k.x), __dmul_rn(k.y, k.y));
  double im = __dadd_rn(__dmul_rn(k.x, k.y), __dmul_rn(k.y, k.x));
  re = __dsub_rn(re, __dmul_rn(alpha, alpha));
  re = __dsub_rn(re, __dmul_rn(beta, beta));
  return cd{re, im};
}

// k^2 and the argument from it and alpha^2, beta^2: the same roundings as kz_arg.
__device__ __forceinline__ cd k_squared(cd k) {
  return cd{__dsub_rn(__dmul_rn(k.x, k.x), __dmul_rn(k.y, k.y)),
            __dadd_rn(__dmul_rn(k.x, k.y), __dmul_rn(k.y, k.x))};
}
__device__ __forceinline__ cd kz_arg_sq(cd kk, double alpha2, double beta2) {
  return cd{__dsub_rn(__dsub_rn(kk.x, alpha2), beta2), kk.y};
}

// alpha = alpha0 + (2 px) pi / 1 ;  beta = beta0 + (2 py) pi / dy
__device__ __forceinline__ void order_ab(int world_1d, double dy, int px, int py, double a0,
                                         double b0, double &alpha, double &beta) {
  alpha = __dadd_rn(a0, __dmul_rn((double)(2 * px), kPi));
  if (world_1d)
    beta = b0;
  else
    beta = __dadd_rn(b0, __ddiv_rn(__dmul_rn((double)(2 * py), kPi), dy));
}

// normalised wavelength wl/period with the Wood-anomaly nudge (mode_calcs.py:41-47)
__device__ __forceinline__ double wl_norm(double wl, double period) {
  double w = wl / period;
  if (fmod(wl, period) == 0.0) w += 1e-10;
  return w;
}

// k = 2 pi n / wl_norm
__device__ __forceinline__ cd wavenumber(cd n, double wln) {
  const double tp = 2.0 * kPi;
  return cd{__ddiv_rn(__dmul_rn(tp, n.x), wln), __ddiv_rn(__dmul_rn(tp, n.y), wln)};
}

struct Fresnel {
  cd R12, T12;
};

// Impedances (backend/mode_calcs.py:199-218) of both polarisations and the
// air/film interface (backend/mode_calcs.py:451-477).
__device__ __forceinline__ void impedances(cd n, cd k, cd kz, cd &zte, cd &ztm) {
  cd zcr = crecip(n);
  cd kokz = cdiv(k, kz);
  zte = cmul(zcr, kokz);
  ztm = cdiv(zcr, kokz);
}

__device__ __forceinline__ Fresnel fresnel(cd z1, cd z2) {
  cd s = cadd(z2, z1);
  Fresnel f;
  f.R12 = cdiv(csub(z2, z1), s);
  f.T12 = cdiv(cmul(cscale(csqrt_p(z2), 2.0), csqrt_p(z1)), s);
  return f;
}

__device__ __forceinline__ cd shear_phase(double alpha, double beta, double c0, double c1, int ncoord) {
  double th = (ncoord == 1) ? __dmul_rn(alpha, c0) : __dadd_rn(__dmul_rn(alpha, c0), __dmul_rn(beta, c1));
  double s, c;
  sincos(th, &s, &c);
  return cd{c, s};
}


}  // namespace emu
