// Batched complex128 GEMM and LU solve entry points (the np.matrix products
// and np.linalg.solve / zgesv calls of backend/stack.py and
// backend/mode_calcs.py, as stand-alone batched kernels).
#include <cuda_runtime.h>

#include "dense_la.cuh"
#include "emu_internal.h"

namespace {

using namespace emu;

struct GemmArgs {
  int m, n, k, lda, ldb, ldc;
  long long sA, sB, sC;
  cd alpha, beta;
  const cd *A;
  const cd *B;
  cd *C;
};

__global__ void __launch_bounds__(kDLThreads) zgemm_batched_kernel(GemmArgs g) {
  __shared__ GemmSmem sm;
  const int b = blockIdx.z;
  cta_gemm_tile(g.m, g.n, g.k, g.alpha, g.A + b * g.sA, g.lda, g.B + b * g.sB, g.ldb, g.beta,
                g.C + b * g.sC, g.ldc, blockIdx.y * kTM, blockIdx.x * kTN, sm);
}

struct GesvArgs {
  int n, nrhs, lda, ldb;
  long long sA, sB;
  cd *A;
  cd *B;
  int *ipiv;
  int *info;
};

__global__ void __launch_bounds__(kDLThreads) zgesv_batched_kernel(GesvArgs g) {
  __shared__ GemmSmem gs;
  __shared__ LuSmem ls;
  const int b = blockIdx.x;
  cd *A = g.A + b * g.sA;
  cd *B = g.B + b * g.sB;
  int *ipiv = g.ipiv + (size_t)b * g.n;
  const int info = cta_getrf(g.n, A, g.lda, ipiv, ls, gs);
  __syncthreads();
  if (g.nrhs > 0) cta_getrs(g.n, g.nrhs, A, g.lda, ipiv, B, g.ldb, gs);
  if (threadIdx.x == 0 && g.info) g.info[b] = info;
}

}  // namespace

extern "C" int emu_zgemm_batched(int m, int n, int k, emu_c128 alpha, const emu_c128 *A, int lda,
                                 long long strideA, const emu_c128 *B, int ldb, long long strideB,
                                 emu_c128 beta, emu_c128 *C, int ldc, long long strideC, int batch,
                                 void *stream) {
  if (m < 0 || n < 0 || k < 0 || batch < 0) return EMU_E_SHAPE;
  if (m == 0 || n == 0 || batch == 0) return EMU_OK;
  if (!A || !B || !C || lda < k || ldb < n || ldc < n) return EMU_E_ARG;
  if (batch > 65535) return EMU_E_SHAPE;
  GemmArgs g{m, n, k, lda, ldb, ldc, strideA, strideB, strideC, cd{alpha.re, alpha.im},
             cd{beta.re, beta.im}, (const cd *)A, (const cd *)B, (cd *)C};
  dim3 grid((n + kTN - 1) / kTN, (m + kTM - 1) / kTM, batch);
  zgemm_batched_kernel<<<grid, kDLThreads, 0, (cudaStream_t)stream>>>(g);
  emu::note_launch();
  return emu::check_launch();
}

extern "C" int emu_zgesv_batched(int n, int nrhs, emu_c128 *A, int lda, long long strideA,
                                 int32_t *ipiv, emu_c128 *B, int ldb, long long strideB,
                                 int32_t *info, int batch, void *stream) {
  if (n < 0 || nrhs < 0 || batch < 0) return EMU_E_SHAPE;
  if (n == 0 || batch == 0) return EMU_OK;
  if (!A || !ipiv || (nrhs > 0 && !B) || lda < n || (nrhs > 0 && ldb < nrhs)) return EMU_E_ARG;
  GesvArgs g{n, nrhs, lda, ldb, strideA, strideB, (cd *)A, (cd *)B, (int *)ipiv, (int *)info};
  zgesv_batched_kernel<<<batch, kDLThreads, 0, (cudaStream_t)stream>>>(g);
  emu::note_launch();
  return emu::check_launch();
}
