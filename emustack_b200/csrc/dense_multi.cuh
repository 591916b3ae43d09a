// Multi-CTA batched dense linear algebra for large interface and cascade
// solves: the same arithmetic as the one-CTA-per-problem routines of
// dense_la.cuh (same tiles, same panel width, same order of operations, so
// results are bit-identical), but every step is its own launch over all
// problems of a batch and spreads each matrix over many CTAs:
//   LU (zgetrf): per panel of kNB columns, one CTA per matrix factors the
//     panel (pivot search, row swaps, rank-1 updates), then a column-parallel
//     unit-lower solve forms U12 and a tiled GEMM updates A22;
//   solve (zgetrs): row interchanges, then blocked forward / backward
//     substitution with column-parallel triangular solves and tiled GEMMs.
// Batched matrices are (base pointer, batch stride in elements, leading
// dimension); problem b is blockIdx.y (.z for the GEMM).
#pragma once
#include <cuda_runtime.h>

#include "dense_la.cuh"
#include "emu_internal.h"

namespace {

using namespace emu;

// ---------------------------------------------------------------- GEMM
struct BGemm {
  int m, n, k;
  cd alpha, beta;
  const cd *A;
  long long sA;
  int lda;
  const cd *B;
  long long sB;
  int ldb;
  cd *C;
  long long sC;
  int ldc;
  const cd *dA;  // optional diagonal scaling of A's columns [b][k]
  long long sdA;
};

__global__ void __launch_bounds__(kDLThreads) bgemm_kernel(BGemm g) {
  __shared__ GemmSmem sm;
  const long long b = blockIdx.z;
  cta_gemm_tile(g.m, g.n, g.k, g.alpha, g.A + b * g.sA, g.lda, g.B + b * g.sB, g.ldb, g.beta,
                g.C + b * g.sC, g.ldc, blockIdx.y * kTM, blockIdx.x * kTN, sm,
                g.dA ? g.dA + b * g.sdA : nullptr, nullptr);
}

inline void bgemm(int m, int n, int k, cd alpha, const cd *A, long long sA, int lda, const cd *B,
                  long long sB, int ldb, cd beta, cd *C, long long sC, int ldc, int batch,
                  cudaStream_t s, const cd *dA = nullptr, long long sdA = 0) {
  if (m <= 0 || n <= 0 || batch <= 0) return;
  BGemm g{m, n, k, alpha, beta, A, sA, lda, B, sB, ldb, C, sC, ldc, dA, sdA};
  dim3 grid((n + kTN - 1) / kTN, (m + kTM - 1) / kTM, batch);
  bgemm_kernel<<<grid, kDLThreads, 0, s>>>(g);
  note_launch();
}

// ---------------------------------------------------------------- LU
// One CTA per matrix: columns j0 .. j0 + jb - 1 of the LU of A (as the
// inner loop of cta_getrf): pivot search, full-row swap, column scaling,
// rank-1 update of the rest of the panel.  info[b] = code + j + 1 for the
// first exactly-zero pivot of this factorisation if info[b] is still 0.
constexpr int kPanelThreads = 1024;
struct PanelSmem {
  double val[kPanelThreads / 32];
  int idx[kPanelThreads / 32];
  int piv;
};

__global__ void __launch_bounds__(kPanelThreads) panel_kernel(cd *A_, long long sA, int lda, int n, int j0,
                                                              int jb, int *ipiv_, long long sip,
                                                              int *info, int code) {
  __shared__ PanelSmem ls;
  const int tid = threadIdx.x, nt = blockDim.x;
  const long long b = blockIdx.x;
  cd *A = A_ + b * sA;
  int *ipiv = ipiv_ + b * sip;
  for (int j = j0; j < j0 + jb; ++j) {
    double best = -1.0;
    int bi = n;
    for (int i = j + tid; i < n; i += nt) {
      const double v = cabs1(A[(size_t)i * lda + j]);
      if (v > best) {
        best = v;
        bi = i;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_down_sync(0xffffffffu, best, o);
      const int oi = __shfl_down_sync(0xffffffffu, bi, o);
      if (ov > best || (ov == best && oi < bi)) {
        best = ov;
        bi = oi;
      }
    }
    if ((tid & 31) == 0) {
      ls.val[tid >> 5] = best;
      ls.idx[tid >> 5] = bi;
    }
    __syncthreads();
    if (tid == 0) {
      double bv = ls.val[0];
      int bx = ls.idx[0];
      for (int w = 1; w < nt / 32; ++w)
        if (ls.val[w] > bv || (ls.val[w] == bv && ls.idx[w] < bx)) {
          bv = ls.val[w];
          bx = ls.idx[w];
        }
      ls.piv = bx;
    }
    __syncthreads();
    const int p = ls.piv;
    if (tid == 0) ipiv[j] = p;
    if (p != j) {
      for (int c = tid; c < n; c += nt) {
        const cd t = A[(size_t)j * lda + c];
        A[(size_t)j * lda + c] = A[(size_t)p * lda + c];
        A[(size_t)p * lda + c] = t;
      }
    }
    __syncthreads();
    const cd ajj = A[(size_t)j * lda + j];
    const bool zero = ajj.x == 0.0 && ajj.y == 0.0;
    if (zero) {
      if (tid == 0 && info && info[b] == 0) info[b] = code + j + 1;
    } else {
      const cd r = crecip(ajj);
      for (int i = j + 1 + tid; i < n; i += nt) A[(size_t)i * lda + j] = cmul(A[(size_t)i * lda + j], r);
    }
    __syncthreads();
    const int pc = j0 + jb - (j + 1);
    if (!zero && pc > 0) {
      const int rows = n - (j + 1);
      for (int e = tid; e < rows * pc; e += nt) {
        const int i = j + 1 + e / pc, c = j + 1 + e % pc;
        A[(size_t)i * lda + c] = csub(A[(size_t)i * lda + c], cmul(A[(size_t)i * lda + j], A[(size_t)j * lda + c]));
      }
    }
    __syncthreads();
  }
}

// X rows r0 .. r0+rb-1 := L11^{-1} X rows (unit lower L11 = L[r0.., r0..],
// rb <= kNB), one thread per column c in [c0, c0 + ncols): the block's L11 is
// staged in shared memory, each column's rb values are held in registers,
// and the substitution runs in the order of cta_getrf / cta_getrs.
__global__ void __launch_bounds__(128) trsm_lower_kernel(const cd *L_, long long sL, int ldl, int r0, int rb,
                                                         cd *X_, long long sX, int ldx, int c0, int ncols) {
  __shared__ cd Ls[kNB][kNB];
  const long long b = blockIdx.y;
  const cd *L = L_ + b * sL;
  cd *X = X_ + b * sX;
  for (int e = threadIdx.x; e < rb * rb; e += blockDim.x) {
    const int r = e / rb, t = e % rb;
    Ls[r][t] = L[(size_t)(r0 + r) * ldl + r0 + t];
  }
  __syncthreads();
  const int cc = blockIdx.x * blockDim.x + threadIdx.x;
  if (cc >= ncols) return;
  const int c = c0 + cc;
  cd x[kNB];
#pragma unroll
  for (int r = 0; r < kNB; ++r)
    if (r < rb) x[r] = X[(size_t)(r0 + r) * ldx + c];
#pragma unroll
  for (int r = 1; r < kNB; ++r) {
    if (r < rb) {
      cd s = x[r];
#pragma unroll
      for (int t = 0; t < r; ++t) s = csub(s, cmul(Ls[r][t], x[t]));
      x[r] = s;
    }
  }
#pragma unroll
  for (int r = 1; r < kNB; ++r)
    if (r < rb) X[(size_t)(r0 + r) * ldx + c] = x[r];
}

// X rows r0 .. r0+rb-1 := U11^{-1} X rows (upper U11 with its diagonal).
__global__ void __launch_bounds__(128) trsm_upper_kernel(const cd *U_, long long sU, int ldu, int r0, int rb,
                                                         cd *X_, long long sX, int ldx, int ncols) {
  __shared__ cd Us[kNB][kNB];
  const long long b = blockIdx.y;
  const cd *U = U_ + b * sU;
  cd *X = X_ + b * sX;
  for (int e = threadIdx.x; e < rb * rb; e += blockDim.x) {
    const int r = e / rb, t = e % rb;
    Us[r][t] = U[(size_t)(r0 + r) * ldu + r0 + t];
  }
  __syncthreads();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncols) return;
  cd x[kNB];
#pragma unroll
  for (int r = 0; r < kNB; ++r)
    if (r < rb) x[r] = X[(size_t)(r0 + r) * ldx + c];
#pragma unroll
  for (int r = kNB - 1; r >= 0; --r) {
    if (r < rb) {
      cd s = x[r];
#pragma unroll
      for (int t = r + 1; t < kNB; ++t)
        if (t < rb) s = csub(s, cmul(Us[r][t], x[t]));
      x[r] = cdiv(s, Us[r][r]);
    }
  }
#pragma unroll
  for (int r = 0; r < kNB; ++r)
    if (r < rb) X[(size_t)(r0 + r) * ldx + c] = x[r];
}

// row interchanges ipiv[0..n) applied in order to the columns of X
__global__ void swap_rows_kernel(cd *X_, long long sX, int ldx, int ncols, const int *ipiv_, long long sip,
                                 int n) {
  const long long b = blockIdx.y;
  cd *X = X_ + b * sX;
  const int *ipiv = ipiv_ + b * sip;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncols; c += gridDim.x * blockDim.x) {
    for (int j = 0; j < n; ++j) {
      const int p = ipiv[j];
      if (p != j) {
        const cd t = X[(size_t)j * ldx + c];
        X[(size_t)j * ldx + c] = X[(size_t)p * ldx + c];
        X[(size_t)p * ldx + c] = t;
      }
    }
  }
}

inline dim3 col_grid(int ncols, int batch) { return dim3((unsigned)((ncols + 127) / 128), (unsigned)batch); }

// In-place LU with partial pivoting of a batch of n x n matrices (cta_getrf's
// arithmetic, spread over CTAs).
inline void getrf_multi(int n, cd *A, long long sA, int lda, int *ipiv, long long sip, int *info, int code,
                        int batch, cudaStream_t s) {
  for (int j0 = 0; j0 < n; j0 += kNB) {
    const int jb = min(kNB, n - j0);
    // a panel is a latency-bound chain of column steps: the widest CTA keeps
    // each step short (the arithmetic does not depend on the width)
    panel_kernel<<<batch, kPanelThreads, 0, s>>>(A, sA, lda, n, j0, jb, ipiv, sip, info, code);
    note_launch();
    const int rest = n - (j0 + jb);
    if (rest > 0) {
      trsm_lower_kernel<<<col_grid(rest, batch), 128, 0, s>>>(A, sA, lda, j0, jb, A, sA, lda, j0 + jb, rest);
      note_launch();
      bgemm(rest, rest, jb, cd{-1.0, 0.0}, A + (size_t)(j0 + jb) * lda + j0, sA, lda,
            A + (size_t)j0 * lda + j0 + jb, sA, lda, cd{1.0, 0.0}, A + (size_t)(j0 + jb) * lda + j0 + jb,
            sA, lda, batch, s);
    }
  }
}

// Solve A X = B in place (B n x nrhs) from getrf_multi's factors.
inline void getrs_multi(int n, int nrhs, const cd *LU, long long sLU, int lda, const int *ipiv, long long sip,
                        cd *B, long long sB, int ldb, int batch, cudaStream_t s) {
  if (nrhs <= 0) return;
  swap_rows_kernel<<<col_grid(nrhs, batch), 128, 0, s>>>(B, sB, ldb, nrhs, ipiv, sip, n);
  note_launch();
  for (int r0 = 0; r0 < n; r0 += kNB) {
    const int rb = min(kNB, n - r0);
    trsm_lower_kernel<<<col_grid(nrhs, batch), 128, 0, s>>>(LU, sLU, lda, r0, rb, B, sB, ldb, 0, nrhs);
    note_launch();
    const int rest = n - (r0 + rb);
    if (rest > 0)
      bgemm(rest, nrhs, rb, cd{-1.0, 0.0}, LU + (size_t)(r0 + rb) * lda + r0, sLU, lda, B + (size_t)r0 * ldb, sB,
            ldb, cd{1.0, 0.0}, B + (size_t)(r0 + rb) * ldb, sB, ldb, batch, s);
  }
  for (int r1 = n; r1 > 0; r1 -= kNB) {
    const int r0 = max(0, r1 - kNB);
    const int rb = r1 - r0;
    trsm_upper_kernel<<<col_grid(nrhs, batch), 128, 0, s>>>(LU, sLU, lda, r0, rb, B, sB, ldb, nrhs);
    note_launch();
    if (r0 > 0)
      bgemm(r0, nrhs, rb, cd{-1.0, 0.0}, LU + r0, sLU, lda, B + (size_t)r0 * ldb, sB, ldb, cd{1.0, 0.0}, B, sB, ldb,
            batch, s);
  }
}

}  // namespace
