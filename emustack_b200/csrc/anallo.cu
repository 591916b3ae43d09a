// Analytic plane-wave modes of homogeneous films (reference: Anallo.calc_kz,
// backend/mode_calcs.py:116-186, and Light._air_ref, backend/objects.py:1745-1777).
//
// One CTA per film/point: every thread owns plane-wave orders; the CTA votes
// on the Wood-anomaly retry, ranks the air sort keys (or applies a given sort
// order) and counts propagating orders.
#include <cuda_runtime.h>

#include "emu_internal.h"
#include "emu_modes.cuh"

namespace {

using namespace emu;
constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) anallo_kernel(EmuAnalloModes p) {
  extern __shared__ __align__(16) unsigned char smem[];
  double *keys = (double *)smem;                     // [Npw]
  __shared__ int s_wood, s_nprop, s_spec;
  const int npw = p.n_pw;
  const double dy = p.period_y / p.period;
  for (int b = blockIdx.x; b < p.n_points; b += gridDim.x) {
    if (threadIdx.x == 0) {
      s_wood = 0;
      s_nprop = 0;
      s_spec = -1;
    }
    __syncthreads();
    const double wln = wl_norm(p.d_wl_nm[b], p.period);
    const emu_c128 nv = p.d_n[b];
    const cd k = wavenumber(cd{nv.re, nv.im}, wln);
    const double a0 = p.d_k_pll[2 * (size_t)b] * p.period;
    const double b0 = p.d_k_pll[2 * (size_t)b + 1] * p.period;
    for (int u = threadIdx.x; u < npw; u += blockDim.x) {
      double al, be;
      order_ab(p.world_1d, dy, p.d_px[u], p.d_py[u], a0, b0, al, be);
      if (cis_zero(csqrt_p(kz_arg(k, al, be)))) s_wood = 1;
    }
    __syncthreads();
    const bool wood = s_wood != 0;
    const double ua0 = wood ? (1 - 1e-9) * a0 : a0, ub0 = wood ? (1 - 1e-9) * b0 : b0;
    for (int u = threadIdx.x; u < npw; u += blockDim.x) {
      double al, be;
      order_ab(p.world_1d, dy, p.d_px[u], p.d_py[u], ua0, ub0, al, be);
      const cd kz = csqrt_p(kz_arg(k, al, be));
      keys[u] = -1 * kz.x + kz.y;
      if (kz.y == 0.0) atomicAdd(&s_nprop, 1);
      if (p.d_alphas) p.d_alphas[(size_t)b * npw + u] = al;
      if (p.d_betas) p.d_betas[(size_t)b * npw + u] = be;
    }
    __syncthreads();
    for (int u = threadIdx.x; u < npw; u += blockDim.x) {
      int r;
      if (p.d_sort_in) {
        // position r holds unsorted order sort_in[r]; find u's position
        r = -1;
        const int32_t *s = p.d_sort_in + (size_t)b * npw;
        for (int v = 0; v < npw; ++v)
          if (s[v] == u) r = v;
      } else {
        const double ku = keys[u];
        r = 0;
        for (int v = 0; v < npw; ++v) {
          const double kv = keys[v];
          r += (kv < ku) || (kv == ku && v < u);
        }
      }
      if (r >= 0) {
        double al, be;
        order_ab(p.world_1d, dy, p.d_px[u], p.d_py[u], ua0, ub0, al, be);
        const cd kz = csqrt_p(kz_arg(k, al, be));
        p.d_kz[(size_t)b * npw + r] = emu_c128{kz.x, kz.y};
        if (p.d_sort_out) p.d_sort_out[(size_t)b * npw + r] = u;
        const bool zero_order = (p.d_px[u] == 0) && (p.world_1d || p.d_py[u] == 0);
        if (zero_order) s_spec = r;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      if (p.d_specular) p.d_specular[b] = s_spec;
      if (p.d_num_prop) p.d_num_prop[b] = s_nprop;
      if (p.d_wood) p.d_wood[b] = s_wood;
    }
    __syncthreads();
  }
}

}  // namespace

extern "C" int emu_anallo_modes(const EmuAnalloModes *p, void *stream) {
  if (!p) return EMU_E_ARG;
  if (p->n_points < 0 || p->n_pw < 1) return EMU_E_SHAPE;
  if (!(p->period > 0) || !(p->period_y > 0)) return EMU_E_ARG;
  if (p->n_points == 0) return EMU_OK;
  if (!p->d_px || !p->d_py || !p->d_wl_nm || !p->d_k_pll || !p->d_n || !p->d_kz) return EMU_E_ARG;
  const size_t smem = sizeof(double) * (size_t)p->n_pw;
  if (smem > 200 * 1024) return EMU_E_SHAPE;
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(anallo_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess)
    return EMU_E_CUDA;
  int grid = p->n_points < 4 * emu::sm_count() ? p->n_points : 4 * emu::sm_count();
  anallo_kernel<<<grid, kThreads, smem, (cudaStream_t)stream>>>(*p);
  emu::note_launch();
  return emu::check_launch();
}
