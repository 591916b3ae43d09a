// Tensor-core GEMM on the 5th-generation tensor cores (tcgen05) with
// split-TF32 operands, for the overlap-integral contraction.
//
//   C[m][n] = sum_k A[m][k] B[n][k]        (both operands K-major, FP32)
//
// computed as Ahi.Bhi + Ahi.Blo + Alo.Bhi, where x = hi + lo with hi, lo
// TF32-rounded (round-to-nearest), accumulated in FP32 in tensor memory
// (TMEM).  Relative error is a few 1e-7 per product (the dropped Alo.Blo
// term is ~2^-22), against ~1e-3 for plain TF32.
//
// One CTA of 128 threads owns a 128 x 128 output tile and a K range (split
// K).  Per K stage of 32: all threads copy the four 128 x 32 operand tiles
// into shared memory in the canonical K-major, no-swizzle UMMA layout (core
// matrices of 8 rows x 16 bytes), fence them to the async proxy, one thread
// issues 4 k-steps x 3 tcgen05.mma (M=128, N=128, K=8) and commits them to
// an mbarrier that every thread waits on (bounded) before the tiles are
// overwritten.  The accumulator is read back with tcgen05.ld (32 lanes x 32
// columns per warp load) and written as FP32 partials of this K split.
//
// Descriptor formats follow the sm100 UMMA definitions (shared-memory matrix
// descriptor: start >> 4, LBO >> 4, SBO >> 4, version 1, layout type;
// instruction descriptor: F32 accumulator, TF32 A/B, K-major, N >> 3, M >> 4).
#include <cuda_runtime.h>
#include <stdint.h>

#include "emu_internal.h"

namespace {

constexpr int kTcM = 128, kTcN = 128, kTcK = 32;  // CTA tile and K stage
constexpr int kTcThreads = 128;
constexpr uint32_t kTmemCols = 128;
constexpr long long kWaitLimit = 1ll << 26;  // bounded mbarrier spins

// bytes of one 128 x 32 FP32 tile in canonical K-major layout
constexpr int kTileBytes = kTcM * kTcK * 4;  // 16 KB

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// canonical K-major no-swizzle offset (bytes) of element (r, k) of a
// 128 x 32 tile: core matrices ordered [k/4][r/8], rows 16 B apart inside.
__device__ __forceinline__ int canon_off(int r, int k) {
  return (((k >> 2) * (kTcM / 8) + (r >> 3)) * 8 + (r & 7)) * 16 + (k & 3) * 4;
}

// Shared-memory matrix descriptor: one MMA reads 128 rows x 8 K-elements =
// 16 row groups x 2 core matrices; LBO = distance between the two K core
// matrices (16 row groups x 128 B), SBO = distance between row groups (128 B).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  const uint64_t lbo = (uint64_t)((kTcM / 8) * 128) >> 4;
  const uint64_t sbo = (uint64_t)128 >> 4;
  return (uint64_t)((saddr >> 4) & 0x3FFF) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

// Instruction descriptor: D F32 (bits 4-5 = 1), A TF32 (7-9 = 2), B TF32
// (10-12 = 2), K-major A and B, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTcN >> 3) << 17) |
                            ((uint32_t)(kTcM >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t"
      ".reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t"
      "}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(phase)
      : "memory");
  return ok != 0;
}

// Bounded wait: returns false (and the caller flags an error) after
// kWaitLimit polls.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
  for (long long i = 0; i < kWaitLimit; ++i)
    if (mbar_try_wait(mbar, phase)) return true;
  return false;
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
        "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
        "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

struct TcArgs {
  const float *Ahi, *Alo, *Bhi, *Blo;  // [Mp][Kp], [Np][Kp]
  int Mp, Np, Kp, kper;                // padded sizes, K per split
  float *C;                            // [splits][Mp][Np]
  int *err;
};

__global__ void __launch_bounds__(kTcThreads, 1) tc_tf32x3_kernel(TcArgs a) {
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  // 4 operand tiles, then the mbarrier and the TMEM address slot
  unsigned char *sm = sm_raw;
  unsigned char *tAhi = sm, *tAlo = sm + kTileBytes, *tBhi = sm + 2 * kTileBytes,
                *tBlo = sm + 3 * kTileBytes;
  uint64_t *mbar = (uint64_t *)(sm + 4 * kTileBytes);
  uint32_t *tslot = (uint32_t *)(sm + 4 * kTileBytes + 16);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * kTcM, n0 = blockIdx.x * kTcN;
  const int split = blockIdx.z;
  const int kbeg = split * a.kper;
  const int kend = min(a.Kp, kbeg + a.kper);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  const uint32_t mb = smem_u32(mbar);
  uint32_t phase = 0;
  bool ok = true;
  int first = 1;
  for (int k0 = kbeg; k0 < kend; k0 += kTcK) {
    // ---- stage the four 128 x 32 tiles (zero outside the padded problem)
    for (int e = tid; e < kTcM * kTcK; e += kTcThreads) {
      const int r = e / kTcK, k = e % kTcK;
      const int off = canon_off(r, k);
      const int gk = k0 + k;
      const bool kin = gk < kend;
      const size_t ia = (size_t)(m0 + r) * a.Kp + gk;
      const size_t ib = (size_t)(n0 + r) * a.Kp + gk;
      const bool ain = kin && (m0 + r) < a.Mp;
      const bool bin = kin && (n0 + r) < a.Np;
      *(float *)(tAhi + off) = ain ? a.Ahi[ia] : 0.0f;
      *(float *)(tAlo + off) = ain ? a.Alo[ia] : 0.0f;
      *(float *)(tBhi + off) = bin ? a.Bhi[ib] : 0.0f;
      *(float *)(tBlo + off) = bin ? a.Blo[ib] : 0.0f;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int s = 0; s < kTcK / 8; ++s) {
        const uint32_t off = (uint32_t)s * 2 * (kTcM / 8) * 128;  // two K core matrices per step
        const uint64_t dAh = smem_desc(smem_u32(tAhi) + off), dAl = smem_desc(smem_u32(tAlo) + off);
        const uint64_t dBh = smem_desc(smem_u32(tBhi) + off), dBl = smem_desc(smem_u32(tBlo) + off);
        mma_tf32(tmem, dAh, dBh, first ? 0u : 1u);
        mma_tf32(tmem, dAh, dBl, 1u);
        mma_tf32(tmem, dAl, dBh, 1u);
        first = 0;
      }
      mma_commit(mb);
    }
    // every thread waits for the MMAs before the tiles are reused
    if (!mbar_wait(mb, phase)) {
      ok = false;
      if (lane == 0) atomicExch(a.err, 1);
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    if (!__syncthreads_and(ok)) break;
    first = 0;
  }
  ok = __syncthreads_and(ok);
  // ---- read the accumulator: warp w owns TMEM lanes (rows) 32w..32w+31
  const int row = m0 + warp * 32 + lane;
  float *Cs = a.C + (size_t)split * a.Mp * a.Np;
  if (kend > kbeg && ok) {
    for (int c0 = 0; c0 < kTcN; c0 += 32) {
      float v[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (row < a.Mp) {
#pragma unroll
        for (int i = 0; i < 32; ++i)
          if (n0 + c0 + i < a.Np) Cs[(size_t)row * a.Np + n0 + c0 + i] = v[i];
      }
    }
  } else if (row < a.Mp) {
    for (int c = 0; c < kTcN; ++c)
      if (n0 + c < a.Np) Cs[(size_t)row * a.Np + n0 + c] = 0.0f;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// x (double) -> hi, lo TF32 values (round to nearest) with x ~ hi + lo
__device__ __forceinline__ void split_tf32(double x, float &hi, float &lo) {
  const float f = (float)x;
  uint32_t h;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(f));
  hi = __uint_as_float(h);
  const float r = (float)(x - (double)hi);
  uint32_t l;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(r));
  lo = __uint_as_float(l);
}

__global__ void split_kernel(const double *x, long long n, float *hi, float *lo) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    split_tf32(x[i], hi[i], lo[i]);
}

__global__ void sum_splits_kernel(const float *C, int splits, long long n, double *out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int p = 0; p < splits; ++p) s += (double)C[(size_t)p * n + i];
    out[i] = s;
  }
}

}  // namespace

namespace emu {

size_t tc_smem_bytes() { return (size_t)4 * kTileBytes + 64; }

// C64[Mp][Np] = A[Mp][Kp] . B[Np][Kp]^T with split-TF32 tensor-core MMAs.
// Operands given as hi/lo FP32 arrays; Cpart scratch [splits][Mp][Np] floats.
int tc_gemm_tf32x3(const float *Ahi, const float *Alo, const float *Bhi, const float *Blo, int Mp,
                   int Np, int Kp, int splits, float *Cpart, double *C64, int *d_err,
                   cudaStream_t s) {
  if (Mp < 1 || Np < 1 || Kp < 1 || splits < 1) return EMU_E_SHAPE;
  const size_t smem = tc_smem_bytes();
  if (cudaFuncSetAttribute(tc_tf32x3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return EMU_E_CUDA;
  int kper = (Kp + splits - 1) / splits;
  kper = (kper + kTcK - 1) / kTcK * kTcK;
  const int used = (Kp + kper - 1) / kper;
  TcArgs ta{Ahi, Alo, Bhi, Blo, Mp, Np, Kp, kper, Cpart, d_err};
  dim3 grid((Np + kTcN - 1) / kTcN, (Mp + kTcM - 1) / kTcM, used);
  tc_tf32x3_kernel<<<grid, kTcThreads, smem, s>>>(ta);
  const long long n = (long long)Mp * Np;
  int g = (int)((n + 255) / 256);
  if (g > 8 * sm_count()) g = 8 * sm_count();
  sum_splits_kernel<<<g, 256, 0, s>>>(Cpart, used, n, C64);
  note_launch(2);
  return check_launch();
}

}  // namespace emu

// Stand-alone entry for testing the tensor-core GEMM: C = A B^T (FP64 in,
// FP64 out, split-TF32 products with FP32 accumulation inside each split).
extern "C" size_t emu_tc_gemm_workspace_size(int m, int n, int k, int splits) {
  if (m < 1 || n < 1 || k < 1 || splits < 1) return 0;
  const size_t a = (size_t)m * k, b = (size_t)n * k;
  return emu::align_up(4 * (2 * a + 2 * b), 256) + emu::align_up(4 * (size_t)splits * m * n, 256) + 256;
}

extern "C" int emu_tc_gemm_tf32x3(int m, int n, int k, const double *d_A, const double *d_B,
                                  double *d_C, int splits, int32_t *d_err, void *d_workspace,
                                  size_t workspace_bytes, void *stream) {
  if (m < 1 || n < 1 || k < 1 || splits < 1) return EMU_E_SHAPE;
  if (!d_A || !d_B || !d_C || !d_err) return EMU_E_ARG;
  if (!d_workspace || workspace_bytes < emu_tc_gemm_workspace_size(m, n, k, splits)) return EMU_E_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  float *w = (float *)d_workspace;
  const size_t a = (size_t)m * k, b = (size_t)n * k;
  float *Ahi = w, *Alo = w + a, *Bhi = w + 2 * a, *Blo = w + 2 * a + b;
  float *Cp = (float *)((char *)d_workspace + emu::align_up(4 * (2 * a + 2 * b), 256));
  const int sms = emu::sm_count();
  split_kernel<<<8 * sms, 256, 0, s>>>(d_A, (long long)a, Ahi, Alo);
  split_kernel<<<8 * sms, 256, 0, s>>>(d_B, (long long)b, Bhi, Blo);
  emu::note_launch(2);
  return emu::tc_gemm_tf32x3(Ahi, Alo, Bhi, Blo, m, n, k, splits, Cp, d_C, (int *)d_err, s);
}
