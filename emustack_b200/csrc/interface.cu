// Interface scattering matrices between a film and a nanostructured layer
// (backend/mode_calcs.py:480-515, r_t_mat_tf_ns), batched, one CTA per
// interface:
//   z = sqrt(1 / Z_film)         A = z o J (P x M)      B = J_dag o z (M x P)
//   G = B A      S = I + G       X = S^-1 B (LU with partial pivoting)
//   R12 = -I + 2 A X   T12 = 2 X   R21 = S^-1 (I - G)   T21 = 2 A S^-1
// and film/film interfaces (backend/mode_calcs.py:451-477), elementwise.
#include <cuda_runtime.h>

#include "dense_la.cuh"
#include "dense_multi.cuh"
#include "emu_internal.h"
#include "emu_modes.cuh"

namespace {

using namespace emu;

struct IfArgs {
  int P, M, npw;
  const cd *kz;    // [b][npw] film k_z (sorted)
  const cd *n;     // [b] film index
  const double *wln;  // [b] normalised wavelength
  const cd *J;     // [b][P][M]
  const cd *Jd;    // [b][M][P]
  cd *R12, *T12, *R21, *T21;
  int *info;
  cd *ws;          // per problem: A (P M), B (M P), S (M M), G (M M), z (P)
  int *ipiv;       // per problem: M
  size_t ws_stride;
};

__device__ __forceinline__ void film_Z(const cd &n, const cd &k, const cd &kz, cd &zte, cd &ztm) {
  cd zcr = crecip(n);
  cd kokz = cdiv(k, kz);
  zte = cmul(zcr, kokz);
  ztm = cdiv(zcr, kokz);
}

__global__ void __launch_bounds__(kDLThreads) interface_dense_kernel(IfArgs a) {
  __shared__ GemmSmem gs;
  __shared__ LuSmem ls;
  const int b = blockIdx.x;
  const int P = a.P, M = a.M, npw = a.npw;
  const int tid = threadIdx.x, nt = blockDim.x;
  cd *ws = a.ws + (size_t)b * a.ws_stride;
  cd *A = ws;
  cd *B = A + (size_t)P * M;
  cd *S = B + (size_t)M * P;
  cd *G = S + (size_t)M * M;
  cd *z = G + (size_t)M * M;
  int *ipiv = a.ipiv + (size_t)b * M;
  const cd *J = a.J + (size_t)b * P * M;
  const cd *Jd = a.Jd + (size_t)b * M * P;
  cd *R12 = a.R12 + (size_t)b * P * P;
  cd *T12 = a.T12 + (size_t)b * M * P;
  cd *R21 = a.R21 + (size_t)b * M * M;
  cd *T21 = a.T21 + (size_t)b * P * M;
  const cd n = a.n[b];
  const cd k = wavenumber(n, a.wln[b]);
  for (int j = tid; j < npw; j += nt) {
    cd zte, ztm;
    film_Z(n, k, a.kz[(size_t)b * npw + j], zte, ztm);
    z[j] = csqrt_p(crecip(zte));
    z[j + npw] = csqrt_p(crecip(ztm));
  }
  __syncthreads();
  for (size_t e = tid; e < (size_t)P * M; e += nt) {
    const int i = (int)(e / M), c = (int)(e % M);
    A[e] = cmul(z[i], J[e]);
  }
  for (size_t e = tid; e < (size_t)M * P; e += nt) {
    const int i = (int)(e % P);
    B[e] = cmul(Jd[e], z[i]);
  }
  __syncthreads();
  // G = B A
  cta_gemm(M, M, P, cd{1.0, 0.0}, B, P, A, M, cd{0.0, 0.0}, G, M, gs);
  __syncthreads();
  for (size_t e = tid; e < (size_t)M * M; e += nt) {
    const int r = (int)(e / M), c = (int)(e % M);
    const cd g = G[e];
    const double one = (r == c) ? 1.0 : 0.0;
    S[e] = cd{one + g.x, 0.0 + g.y};
    R21[e] = cd{one - g.x, 0.0 - g.y};
  }
  for (size_t e = tid; e < (size_t)M * P; e += nt) T12[e] = B[e];
  __syncthreads();
  const int info = cta_getrf(M, S, M, ipiv, ls, gs);
  __syncthreads();
  cta_getrs(M, P, S, M, ipiv, T12, P, gs);      // X = S^-1 B
  cta_getrs(M, M, S, M, ipiv, R21, M, gs);      // R21 = S^-1 (I - G)
  for (size_t e = tid; e < (size_t)M * M; e += nt) {
    const int r = (int)(e / M), c = (int)(e % M);
    G[e] = cd{(r == c) ? 1.0 : 0.0, 0.0};
  }
  __syncthreads();
  cta_getrs(M, M, S, M, ipiv, G, M, gs);        // S^-1
  cta_gemm(P, M, M, cd{2.0, 0.0}, A, M, G, M, cd{0.0, 0.0}, T21, M, gs);
  for (size_t e = tid; e < (size_t)P * P; e += nt) {
    const int r = (int)(e / P), c = (int)(e % P);
    R12[e] = cd{(r == c) ? -1.0 : 0.0, 0.0};
  }
  __syncthreads();
  cta_gemm(P, P, M, cd{2.0, 0.0}, A, M, T12, P, cd{1.0, 0.0}, R12, P, gs);
  __syncthreads();
  for (size_t e = tid; e < (size_t)M * P; e += nt) T12[e] = cscale(T12[e], 2.0);
  if (tid == 0 && a.info) a.info[b] = info;
}

// ---------------------------------------------------------------------------
// Multi-CTA interfaces: interface_dense_kernel's steps, in the same order and
// with the same arithmetic (bit-identical results), each a launch over all
// interfaces of the batch with the matrices spread over many CTAs.

// z = sqrt(1 / Z_film) (both polarisations), A = z o J, B = J_dag o z
__global__ void ifm_prep(IfArgs a) {
  const int P = a.P, M = a.M, npw = a.npw;
  const long long b = blockIdx.y;
  cd *ws = a.ws + b * a.ws_stride;
  cd *A = ws, *B = A + (size_t)P * M;
  const cd n = a.n[b];
  const cd k = wavenumber(n, a.wln[b]);
  // every thread recomputes the z it needs (cheap), so no grid-wide sync
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < 2LL * P * M;
       e += (long long)gridDim.x * blockDim.x) {
    const bool isA = e < (long long)P * M;
    const long long f = isA ? e : e - (long long)P * M;
    const int i = isA ? (int)(f / M) : (int)(f % P);
    const int j = i % npw;
    cd zte, ztm;
    film_Z(n, k, a.kz[b * npw + j], zte, ztm);
    const cd zi = (i < npw) ? csqrt_p(crecip(zte)) : csqrt_p(crecip(ztm));
    if (isA) {
      A[f] = cmul(zi, a.J[b * P * M + f]);
    } else {
      B[f] = cmul(a.Jd[b * M * P + f], zi);
    }
  }
}

// S = I + G, R21 = I - G, T12 = B
__global__ void ifm_sg(IfArgs a) {
  const int P = a.P, M = a.M;
  const long long b = blockIdx.y;
  cd *ws = a.ws + b * a.ws_stride;
  cd *B = ws + (size_t)P * M, *S = B + (size_t)M * P, *G = S + (size_t)M * M;
  cd *R21 = a.R21 + b * M * M, *T12 = a.T12 + b * M * P;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)M * M + (long long)M * P;
       e += (long long)gridDim.x * blockDim.x) {
    if (e < (long long)M * M) {
      const int r = (int)(e / M), c = (int)(e % M);
      const cd g = G[e];
      const double one = (r == c) ? 1.0 : 0.0;
      S[e] = cd{one + g.x, 0.0 + g.y};
      R21[e] = cd{one - g.x, 0.0 - g.y};
    } else {
      const long long f = e - (long long)M * M;
      T12[f] = B[f];
    }
  }
}

// G = I (M x M), R12 = -I (P x P)
__global__ void ifm_eyes(IfArgs a) {
  const int P = a.P, M = a.M;
  const long long b = blockIdx.y;
  cd *G = a.ws + b * a.ws_stride + (size_t)2 * P * M + (size_t)M * M;
  cd *R12 = a.R12 + b * P * P;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)M * M + (long long)P * P;
       e += (long long)gridDim.x * blockDim.x) {
    if (e < (long long)M * M) {
      G[e] = cd{(e / M == e % M) ? 1.0 : 0.0, 0.0};
    } else {
      const long long f = e - (long long)M * M;
      R12[f] = cd{(f / P == f % P) ? -1.0 : 0.0, 0.0};
    }
  }
}

__global__ void ifm_t12x2(IfArgs a) {
  const long long b = blockIdx.y, n = (long long)a.M * a.P;
  cd *T12 = a.T12 + b * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    T12[e] = cscale(T12[e], 2.0);
}

inline dim3 ifm_grid(long long n, int batch) {
  long long g = (n + 255) / 256;
  if (g > 1024) g = 1024;
  return dim3((unsigned)(g < 1 ? 1 : g), (unsigned)batch);
}

int interface_dense_multi(const IfArgs &a, int batch, cudaStream_t s) {
  const int P = a.P, M = a.M;
  const long long S_ = (long long)a.ws_stride;
  cd *A = a.ws, *B = A + (size_t)P * M, *S = B + (size_t)M * P, *G = S + (size_t)M * M;
  const cd one{1.0, 0.0}, zero{0.0, 0.0}, two{2.0, 0.0};
  if (a.info && cudaMemsetAsync(a.info, 0, sizeof(int) * batch, s) != cudaSuccess) return EMU_E_CUDA;
  ifm_prep<<<ifm_grid(2LL * P * M, batch), 256, 0, s>>>(a);
  bgemm(M, M, P, one, B, S_, P, A, S_, M, zero, G, S_, M, batch, s);
  ifm_sg<<<ifm_grid((long long)M * M + (long long)M * P, batch), 256, 0, s>>>(a);
  note_launch(2);
  getrf_multi(M, S, S_, M, a.ipiv, M, a.info, 0, batch, s);
  getrs_multi(M, P, S, S_, M, a.ipiv, M, a.T12, (long long)M * P, P, batch, s);
  getrs_multi(M, M, S, S_, M, a.ipiv, M, a.R21, (long long)M * M, M, batch, s);
  ifm_eyes<<<ifm_grid((long long)M * M + (long long)P * P, batch), 256, 0, s>>>(a);
  note_launch();
  getrs_multi(M, M, S, S_, M, a.ipiv, M, G, S_, M, batch, s);
  bgemm(P, M, M, two, A, S_, M, G, S_, M, zero, a.T21, (long long)P * M, M, batch, s);
  bgemm(P, P, M, two, A, S_, M, a.T12, (long long)M * P, P, one, a.R12, (long long)P * P, P, batch, s);
  ifm_t12x2<<<ifm_grid((long long)M * P, batch), 256, 0, s>>>(a);
  note_launch();
  return check_launch();
}

struct FiArgs {
  int B, npw;
  const cd *kz1, *n1, *kz2, *n2;
  const double *wln;
  cd *R12, *T12;
};

__global__ void film_interface_kernel(FiArgs a) {
  const int P = 2 * a.npw;
  const long long total = (long long)a.B * a.npw;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(e / a.npw), j = (int)(e % a.npw);
    const cd n1 = a.n1[b], n2 = a.n2[b];
    const cd k1 = wavenumber(n1, a.wln[b]), k2 = wavenumber(n2, a.wln[b]);
    cd z1[2], z2[2];
    film_Z(n1, k1, a.kz1[(size_t)b * a.npw + j], z1[0], z1[1]);
    film_Z(n2, k2, a.kz2[(size_t)b * a.npw + j], z2[0], z2[1]);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const cd s = cadd(z2[q], z1[q]);
      a.R12[(size_t)b * P + j + q * a.npw] = cdiv(csub(z2[q], z1[q]), s);
      a.T12[(size_t)b * P + j + q * a.npw] =
          cdiv(cmul(cscale(csqrt_p(z2[q]), 2.0), csqrt_p(z1[q])), s);
    }
  }
}

}  // namespace

extern "C" size_t emu_interface_dense_workspace_size(int batch, int P, int M) {
  if (batch < 0 || P < 1 || M < 1) return 0;
  const size_t per = (size_t)2 * P * M + (size_t)2 * M * M + (size_t)P;
  return (size_t)batch * (per * sizeof(cd) + align_up((size_t)M * sizeof(int), 16)) + 256;
}

extern "C" int emu_interface_dense_batch(int batch, int P, int M, const emu_c128 *d_film_kz,
                                         const emu_c128 *d_film_n, const double *d_wl_norm,
                                         const emu_c128 *d_J, const emu_c128 *d_J_dag,
                                         emu_c128 *d_R12, emu_c128 *d_T12, emu_c128 *d_R21,
                                         emu_c128 *d_T21, int32_t *d_info, void *d_workspace,
                                         size_t workspace_bytes, void *stream) {
  if (batch < 0 || P < 2 || M < 1 || (P % 2)) return EMU_E_SHAPE;
  if (batch == 0) return EMU_OK;
  if (!d_film_kz || !d_film_n || !d_wl_norm || !d_J || !d_J_dag || !d_R12 || !d_T12 || !d_R21 ||
      !d_T21)
    return EMU_E_ARG;
  if (!d_workspace || workspace_bytes < emu_interface_dense_workspace_size(batch, P, M))
    return EMU_E_WORKSPACE;
  IfArgs a;
  a.P = P;
  a.M = M;
  a.npw = P / 2;
  a.kz = (const cd *)d_film_kz;
  a.n = (const cd *)d_film_n;
  a.wln = d_wl_norm;
  a.J = (const cd *)d_J;
  a.Jd = (const cd *)d_J_dag;
  a.R12 = (cd *)d_R12;
  a.T12 = (cd *)d_T12;
  a.R21 = (cd *)d_R21;
  a.T21 = (cd *)d_T21;
  a.info = (int *)d_info;
  a.ws_stride = (size_t)2 * P * M + (size_t)2 * M * M + (size_t)P;
  a.ws = (cd *)d_workspace;
  a.ipiv = (int *)((char *)d_workspace + align_up((size_t)batch * a.ws_stride * sizeof(cd), 16));
  int mode = emu::dense_mode();
  // measured at P = 618, M = 400 (per wavelength of 4 interfaces): with the
  // tensor-core GEMM tile and the cluster LU panel the multi-CTA path wins up
  // to a batch of one interface per SM (1.57 vs 1.79 ms at 148, 1.76 vs
  // 3.61 ms at 64); one CTA per interface beyond that
  if (mode == 0) mode = (M >= 96 && batch <= emu::sm_count()) ? 2 : 1;
  if (mode == 2) return interface_dense_multi(a, batch, (cudaStream_t)stream);
  interface_dense_kernel<<<batch, kDLThreads, 0, (cudaStream_t)stream>>>(a);
  emu::note_launch();
  return emu::check_launch();
}

extern "C" int emu_film_interface_batch(int batch, int n_pw, const emu_c128 *d_kz1,
                                        const emu_c128 *d_n1, const emu_c128 *d_kz2,
                                        const emu_c128 *d_n2, const double *d_wl_norm,
                                        emu_c128 *d_R12, emu_c128 *d_T12, void *stream) {
  if (batch < 0 || n_pw < 1) return EMU_E_SHAPE;
  if (batch == 0) return EMU_OK;
  if (!d_kz1 || !d_n1 || !d_kz2 || !d_n2 || !d_wl_norm || !d_R12 || !d_T12) return EMU_E_ARG;
  FiArgs a{batch, n_pw, (const cd *)d_kz1, (const cd *)d_n1, (const cd *)d_kz2,
           (const cd *)d_n2, d_wl_norm, (cd *)d_R12, (cd *)d_T12};
  const long long total = (long long)batch * n_pw;
  int grid = (int)((total + 255) / 256);
  if (grid > 8 * emu::sm_count()) grid = 8 * emu::sm_count();
  film_interface_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(a);
  emu::note_launch();
  return emu::check_launch();
}
