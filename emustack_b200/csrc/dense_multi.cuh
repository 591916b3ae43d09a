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
#include <algorithm>
#include <cooperative_groups.h>
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

// ---------------------------------------------------------------- cluster panel
// The same panel factorisation by a thread-block cluster of cs <= 8 CTAs
// per matrix: CTA q holds panel rows j0 + q, j0 + q + cs, ... (columns
// j0 .. j0+jb-1) in shared memory.  Per column: each CTA finds its local
// pivot candidate; after a cluster barrier every CTA reads all candidates
// and the pivot row (and the owner of the pivot row reads row j) from the
// other CTAs' shared memory; after a second barrier the rows are swapped
// and every CTA scales and updates its own rows.  Same arithmetic and pivot
// choice as cta_getrf.  The swaps of the columns outside the panel are left
// to laswp_outside_kernel.  Waits are the hardware cluster barrier.
constexpr int kPanelMaxCS = 8;
constexpr int kPanelCTAThreads = 256;
constexpr size_t kPanelMaxSmem = 200 * 1024;

__global__ void __launch_bounds__(kPanelCTAThreads) panel_cluster_kernel(cd *A_, long long sA, int lda, int n,
                                                                         int j0, int jb, int *ipiv_,
                                                                         long long sip, int *info, int code) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char psm[];
  __shared__ double cval[kPanelCTAThreads / 32];
  __shared__ int cidx[kPanelCTAThreads / 32];
  __shared__ double cand_v;  // this CTA's candidate, read by the others
  __shared__ int cand_i;
  __shared__ cd prow[kNB], jrow[kNB];
  const int q = (int)cl.block_rank(), cs = (int)cl.num_blocks();
  const long long b = blockIdx.x / cs;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, w = tid >> 5;
  cd *A = A_ + b * sA;
  int *ipiv = ipiv_ + b * sip;
  const int nr = n - j0;                                  // panel rows
  const int my_rows = nr > q ? (nr - q + cs - 1) / cs : 0;
  cd *Pm = reinterpret_cast<cd *>(psm);                  // [my_rows][kNB]
  auto grow = [&](int l) { return j0 + q + cs * l; };   // local row l -> matrix row
  for (int e = tid; e < my_rows * jb; e += nt) {
    const int l = e / jb, c = e % jb;
    Pm[l * kNB + c] = A[(size_t)grow(l) * lda + j0 + c];
  }
  __syncthreads();
  int first_zero = 0;
  for (int jj = 0; jj < jb; ++jj) {
    const int j = j0 + jj;
    // local pivot candidate among rows >= j (first maximum wins)
    double best = -1.0;
    int bi = n;
    for (int l = tid; l < my_rows; l += nt) {
      const int i = grow(l);
      if (i < j) continue;
      const double v = cabs1(Pm[l * kNB + jj]);
      if (v > best || (v == best && i < bi)) {
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
    if (lane == 0) {
      cval[w] = best;
      cidx[w] = bi;
    }
    __syncthreads();
    if (tid == 0) {
      double bv = cval[0];
      int bx = cidx[0];
      for (int k = 1; k < nt / 32; ++k)
        if (cval[k] > bv || (cval[k] == bv && cidx[k] < bx)) {
          bv = cval[k];
          bx = cidx[k];
        }
      cand_v = bv;
      cand_i = bx;
    }
    cl.sync();  // candidates visible cluster-wide
    // every CTA: the global pivot, then the rows it needs from their owners
    double bv = -1.0;
    int p = n;
    for (int r = 0; r < cs; ++r) {
      const double v = *cl.map_shared_rank(&cand_v, r);
      const int i = *cl.map_shared_rank(&cand_i, r);
      if (v > bv || (v == bv && i < p)) {
        bv = v;
        p = i;
      }
    }
    if (p >= n) p = j;  // no comparable candidate (NaN column): keep the row
    const int qp = (p - j0) % cs, lp = (p - j0) / cs;
    const int qj = (j - j0) % cs, lj = (j - j0) / cs;
    {
      const cd *rp = cl.map_shared_rank(Pm, qp) + (size_t)lp * kNB;
      for (int c = tid; c < jb; c += nt) prow[c] = rp[c];
      if (q == qp && p != j) {
        const cd *rj = cl.map_shared_rank(Pm, qj) + (size_t)lj * kNB;
        for (int c = tid; c < jb; c += nt) jrow[c] = rj[c];
      }
    }
    cl.sync();  // all remote reads done before any row changes
    if (p != j) {
      if (q == qj)
        for (int c = tid; c < jb; c += nt) Pm[lj * kNB + c] = prow[c];
      if (q == qp)
        for (int c = tid; c < jb; c += nt) Pm[lp * kNB + c] = jrow[c];
    }
    if (q == 0 && tid == 0) ipiv[j] = p;
    __syncthreads();
    const cd ajj = prow[jj];
    const bool zero = ajj.x == 0.0 && ajj.y == 0.0;
    if (zero) {
      if (!first_zero) first_zero = j + 1;
    } else {
      const cd r = crecip(ajj);
      const int pc = jb - (jj + 1);
      for (int l = tid; l < my_rows; l += nt) {
        const int i = grow(l);
        if (i <= j) continue;
        const cd lv = cmul(Pm[l * kNB + jj], r);
        Pm[l * kNB + jj] = lv;
        for (int c = jj + 1; c < jj + 1 + pc; ++c) Pm[l * kNB + c] = csub(Pm[l * kNB + c], cmul(lv, prow[c]));
      }
    }
    __syncthreads();
  }
  if (q == 0 && tid == 0 && first_zero && info && info[b] == 0) info[b] = code + first_zero;
  for (int e = tid; e < my_rows * jb; e += nt) {
    const int l = e / jb, c = e % jb;
    A[(size_t)grow(l) * lda + j0 + c] = Pm[l * kNB + c];
  }
  cl.sync();  // no CTA leaves while others may still read its shared memory
}

// The panel's row interchanges ipiv[j0 .. j0+jb) applied in order to the
// columns outside the panel, [0, j0) and [j0+jb, n).
__global__ void laswp_outside_kernel(cd *A_, long long sA, int lda, int n, int j0, int jb, const int *ipiv_,
                                     long long sip) {
  const long long b = blockIdx.y;
  cd *A = A_ + b * sA;
  const int *ipiv = ipiv_ + b * sip;
  const int ncols = n - jb;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ncols; t += gridDim.x * blockDim.x) {
    const int c = t < j0 ? t : t + jb;
    for (int j = j0; j < j0 + jb; ++j) {
      const int p = ipiv[j];
      if (p != j) {
        const cd v = A[(size_t)j * lda + c];
        A[(size_t)j * lda + c] = A[(size_t)p * lda + c];
        A[(size_t)p * lda + c] = v;
      }
    }
  }
}

// The cluster panel's function attributes, set once per device to their
// largest values (kPanelMaxSmem of dynamic shared memory; non-portable
// cluster sizes allowed), never lowered afterwards: host threads that launch
// panels of different sizes at once (two solves on two streams, the server's
// worker threads) then never see a limit another thread set for a smaller
// panel.  Bit 0: the shared-memory limit is set; bit 1: clusters above 8
// CTAs are allowed.  Both threads of a first-call race set the same values.
inline int panel_cluster_attrs() {
  static int state[64] = {};  // 0 = not yet set, else attrs | 4
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
  int st = __atomic_load_n(&state[dev], __ATOMIC_ACQUIRE);
  if (st) return st & 3;
  int attrs = 0;
  if (cudaFuncSetAttribute(panel_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPanelMaxSmem) ==
      cudaSuccess)
    attrs |= 1;
  else
    cudaGetLastError();
  if (cudaFuncSetAttribute(panel_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess)
    attrs |= 2;
  else
    cudaGetLastError();
  __atomic_store_n(&state[dev], attrs | 4, __ATOMIC_RELEASE);
  return attrs;
}

// Launches the cluster panel; false if it would not beat panel_kernel or
// cannot run (the caller then uses panel_kernel).  Cluster size: enough
// CTAs for the panel to fit in shared memory, and as many more (up to 8) as
// keep all clusters of the batch resident at once; a batch that already
// fills the GPU with one wide CTA per matrix keeps panel_kernel.
inline bool panel_cluster(cd *A, long long sA, int lda, int n, int j0, int jb, int *ipiv, long long sip,
                          int *info, int code, int batch, cudaStream_t s, int max_cs = kPanelMaxCS) {
  const size_t row_bytes = (size_t)kNB * sizeof(cd);
  const long long nr = n - j0;
  int cs = 0;
  for (int c = max_cs; c >= 1; --c) {
    const size_t smem = (size_t)((nr + c - 1) / c) * row_bytes;
    if (smem > kPanelMaxSmem) break;
    const long long per_sm = std::min<long long>(2, (long long)(228 * 1024 / (smem + 2048)));
    if ((long long)batch * c <= per_sm * sm_count()) {
      cs = c;
      break;
    }
  }
  if (cs < 2) return false;
  const int attrs = panel_cluster_attrs();
  if (!(attrs & 1)) return false;
  // clusters above 8 CTAs are a non-portable size (the launch fails, and the
  // caller falls back to panel_kernel, where the GPU cannot host them)
  if (cs > 8 && !(attrs & 2)) return false;
  const size_t smem = (size_t)((nr + cs - 1) / cs) * row_bytes;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(batch * cs));
  cfg.blockDim = dim3(kPanelCTAThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (cudaLaunchKernelEx(&cfg, panel_cluster_kernel, A, sA, lda, n, j0, jb, ipiv, sip, info, code) !=
      cudaSuccess)
    return false;
  note_launch();
  const int outside = n - jb;
  if (outside > 0) {
    laswp_outside_kernel<<<dim3((unsigned)((outside + 127) / 128), (unsigned)batch), 128, 0, s>>>(
        A, sA, lda, n, j0, jb, ipiv, sip);
    note_launch();
  }
  return true;
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
  __shared__ cd invd[kNB];
  const long long b = blockIdx.y;
  const cd *U = U_ + b * sU;
  cd *X = X_ + b * sX;
  for (int e = threadIdx.x; e < rb * rb; e += blockDim.x) {
    const int r = e / rb, t = e % rb;
    Us[r][t] = U[(size_t)(r0 + r) * ldu + r0 + t];
  }
  if (threadIdx.x < rb) invd[threadIdx.x] = crecip(U[(size_t)(r0 + threadIdx.x) * ldu + r0 + threadIdx.x]);
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
      x[r] = cmul(s, invd[r]);
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
    // a panel is a latency-bound chain of column steps: a cluster of CTAs
    // keeps the panel in shared memory (one wide CTA through L2 otherwise;
    // the arithmetic is the same)
    if (!panel_cluster(A, sA, lda, n, j0, jb, ipiv, sip, info, code, batch, s)) {
      cudaGetLastError();
      panel_kernel<<<batch, kPanelThreads, 0, s>>>(A, sA, lda, n, j0, jb, ipiv, sip, info, code);
      note_launch();
    }
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
