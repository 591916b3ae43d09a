// CTA-level complex128 dense linear algebra used by the interface and
// cascade kernels: a tiled GEMM update, LU with partial pivoting and the
// triangular solves that go with it.  Matrices are row-major in global
// memory (leading dimension `ld`); one CTA of kDLThreads threads owns a
// problem.  These replace the zgemm / zgesv calls that numpy makes for the
// reference (np.matrix products and np.linalg.solve in backend/stack.py and
// backend/mode_calcs.py).
#pragma once
#include <cuda_runtime.h>

#include "emu_cplx.cuh"

namespace emu {

constexpr int kDLThreads = 256;
constexpr int kTM = 64, kTN = 64, kTK = 8;   // GEMM tile
constexpr int kNB = 32;                      // LU / TRSM block

// Shared tiles of cta_gemm_tile.  A: 64 rows x 8 complex columns stored as
// (re, im) pairs; B: 8 complex rows x 64 complex columns stored as the real
// 16 x 128 matrix [[Re, Im], [-Im, Re]] per element, so that the complex
// product is one real product A_r (m x 2k) * B_r (2k x 2n) whose result,
// read in (re, im) pairs, is the complex C.  Row paddings (+4 doubles) make
// the tensor-core fragment reads free of bank conflicts.
constexpr int kAS = 2 * kTK + 4, kBS = 2 * kTN + 4;
struct GemmSmem {
  double As[kTM][kAS];
  double Bs[2 * kTK][kBS];
};

__device__ __forceinline__ cd ldc(const cd *p) { return *p; }

// D = A B + D on the FP64 tensor cores: one 8 x 8 x 4 product per warp
// (PTX mma.sync m8n8k4 f64; lane l holds A[l/4][l%4], B[l%4][l/4] and
// D[l/4][2(l%4) + {0,1}]).
__device__ __forceinline__ void dmma_884(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// One 64x64 tile of C = alpha * A(m x k) * B(k x n) + beta * C, tile origin
// (r0, c0).  If dA / dB are non-null the rows of A / the rows of B are
// first multiplied by dA[i] / dB[kk] (diagonal factors); conjA conjugates A's
// elements as they are read.  All kDLThreads
// threads of the CTA must call it.  The product runs on the FP64 tensor
// cores: 8 warps in a 2 x 4 grid, each owning a 32 x 32 block of the real
// 64 x 128 result (4 x 4 fragments of 8 x 8).
static __device__ void cta_gemm_tile(int m, int n, int k, cd alpha, const cd *A, int lda, const cd *B,
                              int ldb, cd beta, cd *C, int ldc_, int r0, int c0, GemmSmem &sm,
                              const cd *dA_col = nullptr, const cd *dB_row = nullptr, bool conjA = false) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = warp >> 2, wn = warp & 3;
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  // the next k-tile's elements are fetched into registers while the
  // tensor cores work on the current one
  cd va[2], vb[2];
  auto fetch = [&](int k0) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {  // A: 64 x 8 complex, two elements per thread
      const int r = tid / 8 + 32 * h, c = tid % 8;
      const int gr = r0 + r, gc = k0 + c;
      cd v = cd{0.0, 0.0};
      if (gr < m && gc < k) {
        v = A[(size_t)gr * lda + gc];
        if (conjA) v.y = -v.y;
        if (dA_col) v = cmul(v, dA_col[gc]);
      }
      va[h] = v;
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {  // B: 8 x 64 complex
      const int r = tid / 64 + 4 * h, c = tid % 64;
      const int gr = k0 + r, gc = c0 + c;
      cd v = cd{0.0, 0.0};
      if (gr < k && gc < n) {
        v = B[(size_t)gr * ldb + gc];
        if (dB_row) v = cmul(dB_row[gr], v);
      }
      vb[h] = v;
    }
  };
  if (k > 0) fetch(0);
  for (int k0 = 0; k0 < k; k0 += kTK) {
    // A as (re, im) pairs; B element as the 2 x 2 block [[re, im], [-im, re]]
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int r = tid / 8 + 32 * h, c = tid % 8;
      sm.As[r][2 * c] = va[h].x;
      sm.As[r][2 * c + 1] = va[h].y;
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int r = tid / 64 + 4 * h, c = tid % 64;
      sm.Bs[2 * r][2 * c] = vb[h].x;
      sm.Bs[2 * r][2 * c + 1] = vb[h].y;
      sm.Bs[2 * r + 1][2 * c] = -vb[h].y;
      sm.Bs[2 * r + 1][2 * c + 1] = vb[h].x;
    }
    __syncthreads();
    if (k0 + kTK < k) fetch(k0 + kTK);
#pragma unroll
    for (int ks = 0; ks < 2 * kTK; ks += 4) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = sm.As[wm * 32 + i * 8 + g][ks + t];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = sm.Bs[ks + t][wn * 32 + j * 8 + g];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma_884(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
    __syncthreads();
  }
  const bool zero_beta = beta.x == 0.0 && beta.y == 0.0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int gr = r0 + wm * 32 + i * 8 + g;
    if (gr >= m) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gc = c0 + wn * 16 + j * 4 + t;
      if (gc >= n) continue;
      cd v = cmul(alpha, cd{acc[i][j][0], acc[i][j][1]});
      cd *pc = C + (size_t)gr * ldc_ + gc;
      if (!zero_beta) v = cadd(v, cmul(beta, *pc));
      *pc = v;
    }
  }
}

// C = alpha A B + beta C over all tiles, by one CTA.
static __device__ void cta_gemm(int m, int n, int k, cd alpha, const cd *A, int lda, const cd *B, int ldb,
                         cd beta, cd *C, int ldc_, GemmSmem &sm, const cd *dA_col = nullptr,
                         const cd *dB_row = nullptr) {
  for (int r0 = 0; r0 < m; r0 += kTM)
    for (int c0 = 0; c0 < n; c0 += kTN)
      cta_gemm_tile(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc_, r0, c0, sm, dA_col, dB_row);
}

struct LuSmem {
  double val[kDLThreads / 32];
  int idx[kDLThreads / 32];
  int piv;
  cd rpiv;
};

// |re| + |im| (LAPACK dcabs1, the pivot measure of izamax)
__device__ __forceinline__ double cabs1(cd a) { return fabs(a.x) + fabs(a.y); }

// In-place LU with partial pivoting of the n x n matrix A (row-major), as
// LAPACK zgetrf: A = P L U, unit L below the diagonal, U on and above;
// ipiv[j] = row swapped with j (0-based).  Returns info (0, or j+1 for the
// first exactly-zero pivot; the factorisation continues as LAPACK does).
static __device__ int cta_getrf(int n, cd *A, int lda, int *ipiv, LuSmem &ls, GemmSmem &gs) {
  const int tid = threadIdx.x, nt = blockDim.x;
  int info = 0;
  for (int j0 = 0; j0 < n; j0 += kNB) {
    const int jb = min(kNB, n - j0);
    for (int j = j0; j < j0 + jb; ++j) {
      // pivot search over rows j..n-1 of column j (first maximum wins)
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
        ls.piv = bx < n ? bx : j;  // no comparable candidate (NaN column): keep the row
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
        if (info == 0) info = j + 1;
      } else {
        const cd r = crecip(ajj);
        for (int i = j + 1 + tid; i < n; i += nt) A[(size_t)i * lda + j] = cmul(A[(size_t)i * lda + j], r);
      }
      __syncthreads();
      // rank-1 update of the rest of the panel
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
    const int rest = n - (j0 + jb);
    if (rest > 0) {
      // U12 = L11^{-1} A12 (unit lower), columns in parallel
      for (int c = j0 + jb + tid; c < n; c += nt) {
        for (int r = 1; r < jb; ++r) {
          cd s = A[(size_t)(j0 + r) * lda + c];
          for (int t = 0; t < r; ++t)
            s = csub(s, cmul(A[(size_t)(j0 + r) * lda + j0 + t], A[(size_t)(j0 + t) * lda + c]));
          A[(size_t)(j0 + r) * lda + c] = s;
        }
      }
      __syncthreads();
      // A22 -= L21 U12
      cta_gemm(rest, rest, jb, cd{-1.0, 0.0}, A + (size_t)(j0 + jb) * lda + j0, lda,
               A + (size_t)j0 * lda + j0 + jb, lda, cd{1.0, 0.0},
               A + (size_t)(j0 + jb) * lda + j0 + jb, lda, gs);
      __syncthreads();
    }
  }
  return info;
}

// Solve A X = B in place (B is n x nrhs, ldb) given cta_getrf's output.
static __device__ void cta_getrs(int n, int nrhs, const cd *LU, int lda, const int *ipiv, cd *B, int ldb,
                          GemmSmem &gs) {
  const int tid = threadIdx.x, nt = blockDim.x;
  // row interchanges, in order
  for (int c = tid; c < nrhs; c += nt) {
    for (int j = 0; j < n; ++j) {
      const int p = ipiv[j];
      if (p != j) {
        const cd t = B[(size_t)j * ldb + c];
        B[(size_t)j * ldb + c] = B[(size_t)p * ldb + c];
        B[(size_t)p * ldb + c] = t;
      }
    }
  }
  __syncthreads();
  // forward: unit lower L, blocks of kNB rows
  for (int r0 = 0; r0 < n; r0 += kNB) {
    const int rb = min(kNB, n - r0);
    for (int c = tid; c < nrhs; c += nt) {
      for (int r = 1; r < rb; ++r) {
        cd s = B[(size_t)(r0 + r) * ldb + c];
        for (int t = 0; t < r; ++t) s = csub(s, cmul(LU[(size_t)(r0 + r) * lda + r0 + t], B[(size_t)(r0 + t) * ldb + c]));
        B[(size_t)(r0 + r) * ldb + c] = s;
      }
    }
    __syncthreads();
    const int rest = n - (r0 + rb);
    if (rest > 0) {
      cta_gemm(rest, nrhs, rb, cd{-1.0, 0.0}, LU + (size_t)(r0 + rb) * lda + r0, lda,
               B + (size_t)r0 * ldb, ldb, cd{1.0, 0.0}, B + (size_t)(r0 + rb) * ldb, ldb, gs);
      __syncthreads();
    }
  }
  // backward: upper U, blocks of kNB rows from the bottom
  for (int r1 = n; r1 > 0; r1 -= kNB) {
    const int r0 = max(0, r1 - kNB);
    const int rb = r1 - r0;
    for (int c = tid; c < nrhs; c += nt) {
      for (int r = rb - 1; r >= 0; --r) {
        cd s = B[(size_t)(r0 + r) * ldb + c];
        for (int t = r + 1; t < rb; ++t)
          s = csub(s, cmul(LU[(size_t)(r0 + r) * lda + r0 + t], B[(size_t)(r0 + t) * ldb + c]));
        // the diagonal's reciprocal does not depend on the solve: off the chain
        B[(size_t)(r0 + r) * ldb + c] = cmul(s, crecip(LU[(size_t)(r0 + r) * lda + r0 + r]));
      }
    }
    __syncthreads();
    if (r0 > 0) {
      cta_gemm(r0, nrhs, rb, cd{-1.0, 0.0}, LU + r0, lda, B + (size_t)r0 * ldb, ldb, cd{1.0, 0.0}, B, ldb, gs);
      __syncthreads();
    }
  }
}

}  // namespace emu
