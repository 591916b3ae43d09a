// Refractive indices of the layers of a stack at a batch of wavelengths, on
// the device: the n(lambda) of backend/materials.py:31-186 (Material.n) for
// constant, tabulated and Drude materials, with each layer's loss flag
// applied as backend/mode_calcs.py:186-192 (Anallo.n) applies it.  The
// output is the [B][L] index array the film kernels take, so a sweep over
// wavelengths of tabulated materials never returns to the host between the
// materials and the solve.
//
// Tabulated data are interpolated linearly as scipy.interpolate.interp1d
// (kind 'linear', the reference's choice; scipy 1.18) evaluates it:
//  * real indices (EMU_MAT_TABLE_REAL) through numpy.interp: j the last node
//    with x_j <= x, y = y_j at a node (and at the last node), else
//    y = (y_{j+1} - y_j)/(x_{j+1} - x_j) * (x - x_j) + y_j;
//  * complex indices (EMU_MAT_TABLE) by interp1d's own form: hi =
//    numpy.searchsorted(x, x_new, side='left') clipped to [1, K-1],
//    lo = hi - 1, y = ((x_new - x_lo)/(x_hi - x_lo)) y_hi
//                     + ((x_hi - x_new)/(x_hi - x_lo)) y_lo, termwise.
// Wavelengths outside the table are an error (interp1d's bounds_error),
// reported through d_error and given NaN.
#include <cuda_runtime.h>

#include "emu_cplx.cuh"
#include "emu_internal.h"

namespace {

constexpr int kMaxLayers = 32;

struct MatArgs {
  int n_layers, n_points;
  EmuMaterial mat[kMaxLayers];
  const double *wl;
  emu_c128 *out;
  int32_t *err;
};

__device__ __forceinline__ cd table_n(const EmuMaterial &m, double x, bool &bad) {
  const double *xs = m.d_wl;
  const int K = m.n_rows;
  if (!(x >= xs[0] && x <= xs[K - 1])) {
    bad = true;
    return cd{nan(""), nan("")};
  }
  // first index with xs[i] >= x (searchsorted, side='left')
  int lo = 0, hi = K;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (xs[mid] < x)
      lo = mid + 1;
    else
      hi = mid;
  }
  if (m.kind == EMU_MAT_TABLE_REAL) {
    // numpy.interp: a node gives its value; else the node below and the slope
    if (lo < K && xs[lo] == x) return cd{m.d_n[lo].re, 0.0};
    const int j = lo - 1;  // x_j < x < x_{j+1}
    const double yj = m.d_n[j].re, yk = m.d_n[j + 1].re;
    const double slope = __ddiv_rn(__dsub_rn(yk, yj), __dsub_rn(xs[j + 1], xs[j]));
    return cd{__dadd_rn(__dmul_rn(slope, __dsub_rn(x, xs[j])), yj), 0.0};
  }
  int ihi = lo < 1 ? 1 : (lo > K - 1 ? K - 1 : lo);
  const int ilo = ihi - 1;
  const double xl = xs[ilo], xh = xs[ihi];
  const emu_c128 yl = m.d_n[ilo], yh = m.d_n[ihi];
  const double dx = __dsub_rn(xh, xl);
  const double wh = __ddiv_rn(__dsub_rn(x, xl), dx), wl = __ddiv_rn(__dsub_rn(xh, x), dx);
  return cd{__dadd_rn(__dmul_rn(wh, yh.re), __dmul_rn(wl, yl.re)),
            __dadd_rn(__dmul_rn(wh, yh.im), __dmul_rn(wl, yl.im))};
}

// |z| as the C library's hypot computes it for operands in the normal range
// (glibc 2.35+, Borges' corrected form without fma, "An Improved Algorithm
// for hypot(a,b)", 2019): h = sqrt(ax^2 + ay^2) then one correction step.
// Outside [1e-150, 1e150] the CUDA hypot stands in (ulp-level agreement).
__device__ __forceinline__ double hypot_libc(double x, double y) {
  double ax = fabs(x), ay = fabs(y);
  if (ax < ay) {
    const double t = ax;
    ax = ay;
    ay = t;
  }
  if (!(ax > 1e-150 && ax < 1e150) || !(ay > 1e-150)) return hypot(x, y);
  double h = __dsqrt_rn(__dadd_rn(__dmul_rn(ax, ax), __dmul_rn(ay, ay)));
  double t1, t2;
  if (h <= __dmul_rn(2.0, ay)) {
    const double delta = __dsub_rn(h, ay);
    t1 = __dmul_rn(ax, __dsub_rn(__dmul_rn(2.0, delta), ax));
    t2 = __dmul_rn(__dsub_rn(delta, __dmul_rn(2.0, __dsub_rn(ax, ay))), delta);
  } else {
    const double delta = __dsub_rn(h, ax);
    t1 = __dmul_rn(__dmul_rn(2.0, delta), __dsub_rn(ax, __dmul_rn(2.0, ay)));
    t2 = __dadd_rn(__dmul_rn(__dsub_rn(__dmul_rn(4.0, delta), ay), ay), __dmul_rn(delta, delta));
  }
  return __dsub_rn(h, __ddiv_rn(__dadd_rn(t1, t2), __dmul_rn(2.0, h)));
}

// Principal square root by the steps of the C library's csqrt (numpy.sqrt
// of a complex scalar calls it): d = |z|; for x > 0, r = sqrt((d + x)/2)
// and s = (y/r)/2, else s = sqrt((d - x)/2) and r = |(y/s)/2|; zero real or
// imaginary parts take the closed forms.
__device__ __forceinline__ cd csqrt_libc(cd z) {
  const double x = z.x, y = z.y;
  if (y == 0.0) {
    if (x < 0.0) return cd{0.0, copysign(__dsqrt_rn(-x), y)};
    return cd{fabs(__dsqrt_rn(x)), copysign(0.0, y)};
  }
  if (x == 0.0) {
    const double r = __dsqrt_rn(__dmul_rn(0.5, fabs(y)));
    return cd{r, copysign(r, y)};
  }
  const double d = hypot_libc(x, y);
  double r, s;
  if (x > 0.0) {
    r = __dsqrt_rn(__dmul_rn(0.5, __dadd_rn(d, x)));
    s = __dmul_rn(0.5, __ddiv_rn(y, r));
  } else {
    s = __dsqrt_rn(__dmul_rn(0.5, __dsub_rn(d, x)));
    r = fabs(__dmul_rn(0.5, __ddiv_rn(y, s)));
  }
  return cd{r, copysign(s, y)};
}

// a / b as numpy divides complex numbers (Smith's method with the reciprocal
// of the scaled denominator taken once).
__device__ __forceinline__ cd cdiv_numpy(cd a, cd b) {
  if (fabs(b.x) >= fabs(b.y)) {
    if (b.x == 0.0 && b.y == 0.0) return cdiv(a, b);
    const double rat = __ddiv_rn(b.y, b.x);
    const double scl = __ddiv_rn(1.0, __dadd_rn(b.x, __dmul_rn(b.y, rat)));
    return cd{__dmul_rn(__dadd_rn(a.x, __dmul_rn(a.y, rat)), scl),
              __dmul_rn(__dsub_rn(a.y, __dmul_rn(a.x, rat)), scl)};
  }
  const double rat = __ddiv_rn(b.x, b.y);
  const double scl = __ddiv_rn(1.0, __dadd_rn(b.y, __dmul_rn(b.x, rat)));
  return cd{__dmul_rn(__dadd_rn(__dmul_rn(a.x, rat), a.y), scl),
            __dmul_rn(__dsub_rn(__dmul_rn(a.y, rat), a.x), scl)};
}

// sqrt(eps_inf - wp^2 / (w^2 + i wg w)), w = 2 pi c / (wl 1e-9), with the
// reference's order of operations (materials.py:140-146) and numpy's
// complex arithmetic: the imaginary part of the denominator is
// (wg 2 pi c) / (wl 1e-9), the quotient is numpy's complex division and the
// root the C library's csqrt, so the result is numpy's to the bit except
// where numpy's w**2 (the C library's pow) rounds w^2 to the other
// neighbour of the exact square, which w*w here does not.
__device__ __forceinline__ cd drude_n(const EmuMaterial &m, double wl) {
  const double c = 299792458.0;
  const double wp = m.drude[0], wg = m.drude[1], eps_inf = m.drude[2];
  const double a = __dmul_rn(2.0 * 3.141592653589793, c), t = __dmul_rn(wl, 1e-9);
  const double w = __ddiv_rn(a, t);
  const cd den{__dmul_rn(w, w), __ddiv_rn(__dmul_rn(wg, a), t)};
  const cd q = cdiv_numpy(cd{__dmul_rn(wp, wp), 0.0}, den);
  return csqrt_libc(cd{__dsub_rn(eps_inf, q.x), __dsub_rn(0.0, q.y)});
}

__global__ void material_kernel(MatArgs a) {
  const long long total = (long long)a.n_points * a.n_layers;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(i / a.n_layers), l = (int)(i % a.n_layers);
    const EmuMaterial &m = a.mat[l];
    const double wl = a.wl[b];
    bool bad = false;
    cd n;
    if (m.kind == EMU_MAT_TABLE || m.kind == EMU_MAT_TABLE_REAL)
      n = table_n(m, wl, bad);
    else if (m.kind == EMU_MAT_DRUDE)
      n = drude_n(m, wl);
    else
      n = cd{m.n_const.re, m.n_const.im};
    if (!m.loss) n.y = 0.0;
    if (bad && a.err) atomicExch(a.err, 1);
    a.out[i] = emu_c128{n.x, n.y};
  }
}

}  // namespace

extern "C" int emu_material_n_batch(const EmuMaterial *h_materials, int n_layers, int n_points,
                                    const double *d_wl_nm, emu_c128 *d_n, int32_t *d_error,
                                    void *stream) {
  if (!h_materials || n_layers < 1 || n_layers > kMaxLayers || n_points < 0) return EMU_E_ARG;
  if (n_points == 0) return EMU_OK;
  if (!d_wl_nm || !d_n) return EMU_E_ARG;
  MatArgs a;
  a.n_layers = n_layers;
  a.n_points = n_points;
  for (int l = 0; l < n_layers; ++l) {
    const EmuMaterial &m = h_materials[l];
    if (m.kind < EMU_MAT_CONSTANT || m.kind > EMU_MAT_TABLE_REAL) return EMU_E_ARG;
    if ((m.kind == EMU_MAT_TABLE || m.kind == EMU_MAT_TABLE_REAL) && (m.n_rows < 2 || !m.d_wl || !m.d_n))
      return EMU_E_ARG;
    a.mat[l] = m;
  }
  a.wl = d_wl_nm;
  a.out = d_n;
  a.err = d_error;
  const long long total = (long long)n_points * n_layers;
  long long blocks = (total + 255) / 256;
  const long long cap = 8LL * emu::sm_count();
  if (blocks > cap) blocks = cap;
  material_kernel<<<(int)blocks, 256, 0, (cudaStream_t)stream>>>(a);
  emu::note_launch();
  return emu::check_launch();
}
