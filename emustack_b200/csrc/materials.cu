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

// sqrt(eps_inf - wp^2 / (w^2 + i wg w)), w = 2 pi c / (wl 1e-9), with the
// reference's order of operations (materials.py:140-146): the imaginary
// part of the denominator is (wg 2 pi c) / (wl 1e-9)
__device__ __forceinline__ cd drude_n(const EmuMaterial &m, double wl) {
  const double c = 299792458.0;
  const double wp = m.drude[0], wg = m.drude[1], eps_inf = m.drude[2];
  const double a = __dmul_rn(2.0 * 3.141592653589793, c), t = __dmul_rn(wl, 1e-9);
  const double w = __ddiv_rn(a, t);
  const cd den{__dmul_rn(w, w), __ddiv_rn(__dmul_rn(wg, a), t)};
  const cd q = cdiv(cd{__dmul_rn(wp, wp), 0.0}, den);
  return csqrt_p(cd{__dsub_rn(eps_inf, q.x), -q.y});
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
