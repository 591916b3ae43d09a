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
// K).  The four 128 x 32 operand tiles of each K stage arrive by TMA in the
// canonical K-major, no-swizzle UMMA layout (core matrices of 8 rows x 16
// bytes) through a 3-stage mbarrier pipeline; one thread issues 4 k-steps x
// 3 tcgen05.mma (M=128, N=128, K=8) per stage.  The accumulator is read back
// with tcgen05.ld (32 lanes x 32 columns per warp load) and written as FP32
// partials of this K split.  Every mbarrier wait is bounded.
//
// Descriptor formats follow the sm100 UMMA definitions (shared-memory matrix
// descriptor: start >> 4, LBO >> 4, SBO >> 4, version 1, layout type;
// instruction descriptor: F32 accumulator, TF32 A/B, K-major, N >> 3, M >> 4).
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
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

// ---------------------------------------------------------------------------
// TMA-fed, 3-stage pipelined variant.  Warp 0 lane 0 streams the four
// operand tiles of each K stage into shared memory with cp.async.bulk.tensor
// (a box of 4 FP32 x 128 rows per 16-byte K chunk lands exactly in the
// canonical K-major no-swizzle layout), completing on full[stage]; warp 1
// lane 0 issues the 12 MMAs of a stage once full[stage] completes and
// commits them to empty[stage], which frees the buffer for the producer.
constexpr int kStages = 3;
constexpr int kStageBytes = 4 * kTileBytes;  // 64 KB

struct TmaMaps {
  CUtensorMap ahi, alo, bhi, blo;
};

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
      ::"r"(dst), "l"((uint64_t)map), "r"(mbar), "r"(x), "r"(y)
      : "memory");
}

__global__ void __launch_bounds__(kTcThreads, 1)
    tc_tf32x3_tma_kernel(const __grid_constant__ TmaMaps maps, int Mp, int Np, int Kp, int kper, float *C,
                         int *err) {
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  unsigned char *buf = sm_raw;  // kStages x 64 KB
  uint64_t *bars = (uint64_t *)(sm_raw + kStages * kStageBytes);
  uint32_t *tslot = (uint32_t *)(bars + 2 * kStages + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * kTcM, n0 = blockIdx.x * kTcN;
  const int split = blockIdx.z;
  const int kbeg = split * kper;
  const int kend = min(Kp, kbeg + kper);
  const int nst = kend > kbeg ? (kend - kbeg + kTcK - 1) / kTcK : 0;
  const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + kStages), done = smem_u32(bars + 2 * kStages);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int i = 0; i < kStages; ++i) {
      mbar_init(full0 + 8 * i, 1);
      mbar_init(empty0 + 8 * i, 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  bool ok = true;

  if (warp == 0 && lane == 0) {
    // ---- producer
    for (int t = 0; t < nst && ok; ++t) {
      const int b = t % kStages;
      if (t >= kStages && !mbar_wait(empty0 + 8 * b, (uint32_t)((t / kStages - 1) & 1))) {
        ok = false;
        break;
      }
      const uint32_t fb = full0 + 8 * b;
      mbar_expect_tx(fb, (uint32_t)kStageBytes);
      const uint32_t base = smem_u32(buf + (size_t)b * kStageBytes);
      const int k0 = kbeg + t * kTcK;
#pragma unroll
      for (int kc = 0; kc < kTcK / 4; ++kc) {
        const int x = k0 + 4 * kc;
        const uint32_t o = (uint32_t)kc * (kTcM / 8) * 128;
        tma_load_2d(base + 0 * kTileBytes + o, &maps.ahi, x, m0, fb);
        tma_load_2d(base + 1 * kTileBytes + o, &maps.alo, x, m0, fb);
        tma_load_2d(base + 2 * kTileBytes + o, &maps.bhi, x, n0, fb);
        tma_load_2d(base + 3 * kTileBytes + o, &maps.blo, x, n0, fb);
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer
    for (int t = 0; t < nst && ok; ++t) {
      const int b = t % kStages;
      if (!mbar_wait(full0 + 8 * b, (uint32_t)((t / kStages) & 1))) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t base = smem_u32(buf + (size_t)b * kStageBytes);
#pragma unroll
      for (int s = 0; s < kTcK / 8; ++s) {
        const uint32_t off = (uint32_t)s * 2 * (kTcM / 8) * 128;
        const uint64_t dAh = smem_desc(base + 0 * kTileBytes + off), dAl = smem_desc(base + 1 * kTileBytes + off);
        const uint64_t dBh = smem_desc(base + 2 * kTileBytes + off), dBl = smem_desc(base + 3 * kTileBytes + off);
        mma_tf32(tmem, dAh, dBh, (t == 0 && s == 0) ? 0u : 1u);
        mma_tf32(tmem, dAh, dBl, 1u);
        mma_tf32(tmem, dAl, dBh, 1u);
      }
      mma_commit(empty0 + 8 * b);
    }
    if (nst > 0) mma_commit(done);
  }
  __syncwarp();
  if (!ok) atomicExch(err, 1);
  // ---- epilogue: wait for the last MMAs (bounded), then TMEM -> registers -> global
  bool fin = (nst == 0) || mbar_wait(done, 0);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  fin = __syncthreads_and(fin && ok);
  if (!fin && tid == 0) atomicExch(err, 1);
  const int row = m0 + warp * 32 + lane;
  float *Cs = C + (size_t)split * Mp * Np;
  if (nst > 0 && fin) {
    for (int c0 = 0; c0 < kTcN; c0 += 32) {
      float v[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (row < Mp) {
#pragma unroll
        for (int i = 0; i < 32; ++i)
          if (n0 + c0 + i < Np) Cs[(size_t)row * Np + n0 + c0 + i] = v[i];
      }
    }
  } else if (row < Mp) {
    for (int c = 0; c < kTcN; ++c)
      if (n0 + c < Np) Cs[(size_t)row * Np + n0 + c] = 0.0f;
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

// rows x k (row-major FP64) -> rows x k4 hi/lo, zero padded to k4 columns
__global__ void split_pad_kernel(const double *x, int rows, int k, int k4, float *hi, float *lo) {
  const long long n = (long long)rows * k4;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long r = i / k4, c = i % k4;
    if (c < k) {
      split_tf32(x[r * k + c], hi[i], lo[i]);
    } else {
      hi[i] = 0.0f;
      lo[i] = 0.0f;
    }
  }
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

// C64[Mp][Np] = A[Mp][Kp] . B[Np][Kp]^T with split-TF32 tensor-core MMAs.
// Operands given as hi/lo FP32 arrays; Cpart scratch [splits][Mp][Np] floats.
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

// 2D map over a row-major [rows][Kp] FP32 matrix, box = 4 (K) x 128 (rows).
static bool make_map(CUtensorMap *m, const float *ptr, int rows, int Kp) {
  auto fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)Kp * 4};
  const cuuint32_t box[2] = {4, (cuuint32_t)kTcM};
  const cuuint32_t estr[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)ptr, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

size_t tc_smem_bytes() { return (size_t)kStages * kStageBytes + 128; }

// C64[Mp][Np] = A[Mp][Kp] . B[Np][Kp]^T with split-TF32 tensor-core MMAs.
// Operands given as hi/lo FP32 arrays (16-byte aligned, Kp % 4 == 0);
// Cpart scratch [splits][Mp][Np] floats.
int tc_gemm_tf32x3(const float *Ahi, const float *Alo, const float *Bhi, const float *Blo, int Mp,
                   int Np, int Kp, int splits, float *Cpart, double *C64, int *d_err,
                   cudaStream_t s) {
  if (Mp < 1 || Np < 1 || Kp < 4 || splits < 1 || (Kp % 4)) return EMU_E_SHAPE;
  TmaMaps maps;
  if (!make_map(&maps.ahi, Ahi, Mp, Kp) || !make_map(&maps.alo, Alo, Mp, Kp) ||
      !make_map(&maps.bhi, Bhi, Np, Kp) || !make_map(&maps.blo, Blo, Np, Kp))
    return EMU_E_CUDA;
  const size_t smem = tc_smem_bytes();
  if (cudaFuncSetAttribute(tc_tf32x3_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return EMU_E_CUDA;
  int kper = (Kp + splits - 1) / splits;
  kper = (kper + kTcK - 1) / kTcK * kTcK;
  const int used = (Kp + kper - 1) / kper;
  dim3 grid((Np + kTcN - 1) / kTcN, (Mp + kTcM - 1) / kTcM, used);
  tc_tf32x3_tma_kernel<<<grid, kTcThreads, smem, s>>>(maps, Mp, Np, Kp, kper, Cpart, d_err);
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
  const size_t k4 = (size_t)(k + 3) / 4 * 4;
  const size_t a = (size_t)m * k4, b = (size_t)n * k4;
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
  const int k4 = (k + 3) / 4 * 4;
  const size_t a = (size_t)m * k4, b = (size_t)n * k4;
  float *Ahi = w, *Alo = w + a, *Bhi = w + 2 * a, *Blo = w + 2 * a + b;
  float *Cp = (float *)((char *)d_workspace + emu::align_up(4 * (2 * a + 2 * b), 256));
  const int sms = emu::sm_count();
  split_pad_kernel<<<8 * sms, 256, 0, s>>>(d_A, m, k, k4, Ahi, Alo);
  split_pad_kernel<<<8 * sms, 256, 0, s>>>(d_B, n, k, k4, Bhi, Blo);
  emu::note_launch(2);
  return emu::tc_gemm_tf32x3(Ahi, Alo, Bhi, Blo, m, n, k4, splits, Cp, d_C, (int *)d_err, s);
}
