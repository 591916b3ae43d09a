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
// One CTA of 192 threads owns a 128 x 256 output tile and a K range (split
// K).  Per K stage of 32 FP32 values (one 128-byte row per operand row):
//   warp 0 (one lane) loads the A (128 x 32) and B (256 x 32) FP32 tiles by
//     TMA with 128-byte swizzling, completing on full[stage];
//   warps 2-5 split them in shared memory: hi = rna_tf32(x) in place and
//     lo = rna_tf32(x - hi) into a twin tile at the same offsets (an
//     elementwise pass, so the swizzled layout carries over), then make the
//     writes visible to the tensor core (proxy fence) and arrive on
//     split[stage];
//   warp 1 (one lane) issues 4 k-steps x 3 tcgen05.mma (M=128, N=256, K=8)
//     per stage and commits them to empty[stage], freeing the buffers.
// Only x travels from memory (half the bytes of precomputed hi/lo pairs).
// The tensor cores accumulate in FP32 with a bias that grows with the K
// range of one accumulation (about -6e-9 x K relative), so each
// accumulation covers one chunk of 256 K values (8 stages) and starts from
// zero: after a chunk's MMAs (committed to acc_full), warps 2-5 read the
// accumulator with tcgen05.ld (each warp its 32-lane quarter of TMEM), add
// the running sum of the earlier chunks held in the other half of TMEM
// (FP32, round to nearest) and store it back with tcgen05.st, then free the
// accumulator (acc_empty) for the next chunk; after the last chunk they write
// the CTA's sum as the FP32 partial of this K split.  Every mbarrier wait is
// bounded.
//
// Descriptor formats follow the sm100 UMMA definitions (shared-memory matrix
// descriptor: start >> 4, LBO >> 4, SBO >> 4, version 1, layout type
// SWIZZLE_128B; instruction descriptor: F32 accumulator, TF32 A/B, K-major,
// N >> 3, M >> 4).
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include "emu_internal.h"

namespace {

constexpr int kTcM = 128, kTcN = 256, kTcK = 32;  // CTA tile and K stage (32 FP32 = 128 B)
constexpr int kTcThreads = 192;
constexpr int kSplitThreads = 128;                  // warps 2-5
constexpr uint32_t kTmemCols = 512;  // accumulator [0, 256), running sum [256, 512)
constexpr int kChunkStages = 8;       // K stages per tensor-memory accumulation (256 values)
constexpr long long kWaitLimit = 1ll << 26;  // bounded mbarrier spins

constexpr int kATileBytes = kTcM * kTcK * 4;  // 16 KB
constexpr int kBTileBytes = kTcN * kTcK * 4;  // 32 KB
// stage: [A x/hi][A lo][B x/hi][B lo]
constexpr int kStageBytes = 2 * kATileBytes + 2 * kBTileBytes;  // 96 KB
constexpr int kStages = 2;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor for a K-major operand in the 128-byte
// swizzled layout TMA writes: rows of 128 B, 8-row atoms of 1024 B (SBO), LBO
// unused (1), layout type 2 (SWIZZLE_128B) in bits 61-63.  The K-step s of
// a stage starts s * 32 bytes into the (1024-byte aligned) tile.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t saddr) {
  const uint64_t lbo = 1;
  const uint64_t sbo = (uint64_t)1024 >> 4;
  return (uint64_t)((saddr >> 4) & 0x3FFF) | (lbo << 16) | (sbo << 32) | (1ull << 46) | (2ull << 61);
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

__device__ __forceinline__ void tmem_st32(uint32_t taddr, const float *v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
      "{%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, "
      "%17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};\n" ::"r"(taddr),
      "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
      "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
      "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
      "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
      "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
      "r"(__float_as_uint(v[15])), "r"(__float_as_uint(v[16])), "r"(__float_as_uint(v[17])),
      "r"(__float_as_uint(v[18])), "r"(__float_as_uint(v[19])), "r"(__float_as_uint(v[20])),
      "r"(__float_as_uint(v[21])), "r"(__float_as_uint(v[22])), "r"(__float_as_uint(v[23])),
      "r"(__float_as_uint(v[24])), "r"(__float_as_uint(v[25])), "r"(__float_as_uint(v[26])),
      "r"(__float_as_uint(v[27])), "r"(__float_as_uint(v[28])), "r"(__float_as_uint(v[29])),
      "r"(__float_as_uint(v[30])), "r"(__float_as_uint(v[31]))
      : "memory");
}

struct TmaMaps {
  CUtensorMap a, b;
};

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

// box at (x = K, y = row, z = problem) of a 3D [batch][rows][Kp] map
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, int x, int y, int z,
                                            uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
      ::"r"(dst), "l"((uint64_t)map), "r"(mbar), "r"(x), "r"(y), "r"(z)
      : "memory");
}

__device__ __forceinline__ float rna_tf32(float x) {
  uint32_t h;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
  return __uint_as_float(h);
}

// In-place hi and twin-tile lo of n4 float4 values.
__device__ __forceinline__ void split_tile(float4 *x, float4 *lo, int n4, int t) {
  for (int i = t; i < n4; i += kSplitThreads) {
    const float4 v = x[i];
    float4 h, l;
    h.x = rna_tf32(v.x);
    h.y = rna_tf32(v.y);
    h.z = rna_tf32(v.z);
    h.w = rna_tf32(v.w);
    l.x = rna_tf32(v.x - h.x);
    l.y = rna_tf32(v.y - h.y);
    l.z = rna_tf32(v.z - h.z);
    l.w = rna_tf32(v.w - h.w);
    x[i] = h;
    lo[i] = l;
  }
}

__global__ void __launch_bounds__(kTcThreads, 1)
    tc_tf32x3_kernel(const __grid_constant__ TmaMaps maps, int Mp, int Np, int Kp, int kper, int nsplit,
                     float *C, int *err) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  // 128-byte swizzled tiles need 1024-byte aligned shared addresses
  const uint32_t raw = smem_u32(sm_raw);
  unsigned char *buf = sm_raw + (((raw + 1023u) & ~1023u) - raw);
  uint64_t *bars = (uint64_t *)(buf + kStages * kStageBytes);
  uint32_t *tslot = (uint32_t *)(bars + 3 * kStages + 3);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * kTcM, n0 = blockIdx.x * kTcN;
  const int split = blockIdx.z % nsplit, prob = blockIdx.z / nsplit;
  const int kbeg = split * kper;
  const int kend = min(Kp, kbeg + kper);
  const int nst = kend > kbeg ? (kend - kbeg + kTcK - 1) / kTcK : 0;
  const uint32_t full0 = smem_u32(bars), spl0 = smem_u32(bars + kStages),
                 empty0 = smem_u32(bars + 2 * kStages), acc_full = smem_u32(bars + 3 * kStages),
                 acc_empty = smem_u32(bars + 3 * kStages + 1), done = smem_u32(bars + 3 * kStages + 2);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int i = 0; i < kStages; ++i) {
      mbar_init(full0 + 8 * i, 1);
      mbar_init(spl0 + 8 * i, kSplitThreads);
      mbar_init(empty0 + 8 * i, 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, kSplitThreads);
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  bool ok = true;

  if (warp == 0) {
    if (lane == 0) {
      // ---- producer: x tiles of A and B by TMA
      for (int t = 0; t < nst; ++t) {
        const int b = t % kStages;
        if (t >= kStages && !mbar_wait(empty0 + 8 * b, (uint32_t)((t / kStages - 1) & 1))) {
          ok = false;
          break;
        }
        const uint32_t fb = full0 + 8 * b;
        mbar_expect_tx(fb, (uint32_t)(kATileBytes + kBTileBytes));
        const uint32_t base = smem_u32(buf + (size_t)b * kStageBytes);
        const int k0 = kbeg + t * kTcK;
        tma_load_3d(base, &maps.a, k0, m0, prob, fb);
        tma_load_3d(base + 2 * kATileBytes, &maps.b, k0, n0, prob, fb);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ---- MMA issuer
      for (int t = 0; t < nst; ++t) {
        const int b = t % kStages, j = t % kChunkStages, c = t / kChunkStages;
        // a new chunk starts once the epilogue has taken the previous one
        if (j == 0 && c > 0 && !mbar_wait(acc_empty, (uint32_t)((c - 1) & 1))) {
          ok = false;
          break;
        }
        if (!mbar_wait(spl0 + 8 * b, (uint32_t)((t / kStages) & 1))) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t base = smem_u32(buf + (size_t)b * kStageBytes);
        const uint32_t ah = base, al = base + kATileBytes;
        const uint32_t bh = base + 2 * kATileBytes, bl = bh + kBTileBytes;
#pragma unroll
        for (int k = 0; k < kTcK / 8; ++k) {
          const uint32_t o = (uint32_t)k * 32;
          const uint64_t dAh = smem_desc_sw128(ah + o), dAl = smem_desc_sw128(al + o);
          const uint64_t dBh = smem_desc_sw128(bh + o), dBl = smem_desc_sw128(bl + o);
          mma_tf32(tmem, dAh, dBh, (j == 0 && k == 0) ? 0u : 1u);
          mma_tf32(tmem, dAh, dBl, 1u);
          mma_tf32(tmem, dAl, dBh, 1u);
        }
        mma_commit(empty0 + 8 * b);
        if (j == kChunkStages - 1 || t == nst - 1) mma_commit(acc_full);
      }
      // tracks every MMA issued above, also when a wait gave up: tensor
      // memory is freed only after they have completed
      if (nst > 0) mma_commit(done);
    }
  } else {
    // ---- splitters and epilogue (warps 2-5)
    const int st = tid - 64;
    const int q = warp & 3;  // TMEM lane quarter this warp may read
    const int row = m0 + q * 32 + lane;
    float *Cs = C + ((size_t)prob * nsplit + split) * Mp * Np;
    const uint32_t tacc = tmem + ((uint32_t)(q * 32) << 16), trun = tacc + 256;
    for (int t = 0; t < nst; ++t) {
      const int b = t % kStages, j = t % kChunkStages, c = t / kChunkStages;
      // warp-uniform outcomes: the tcgen05.ld / st below need converged warps
      if (!__all_sync(0xffffffffu, mbar_wait(full0 + 8 * b, (uint32_t)((t / kStages) & 1)))) {
        ok = false;
        break;
      }
      unsigned char *base = buf + (size_t)b * kStageBytes;
      split_tile((float4 *)base, (float4 *)(base + kATileBytes), kATileBytes / 16, st);
      split_tile((float4 *)(base + 2 * kATileBytes), (float4 *)(base + 2 * kATileBytes + kBTileBytes),
                 kBTileBytes / 16, st);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(spl0 + 8 * b);
      if (j != kChunkStages - 1 && t != nst - 1) continue;
      // end of a chunk: fold its accumulator into the running sum
      if (!__all_sync(0xffffffffu, mbar_wait(acc_full, (uint32_t)(c & 1)))) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const bool last = t == nst - 1;
      for (int c0 = 0; c0 < kTcN; c0 += 32) {
        float v[32];
        tmem_ld32(tacc + (uint32_t)c0, v);
        if (c > 0) {
          float r[32];
          tmem_ld32(trun + (uint32_t)c0, r);
#pragma unroll
          for (int i = 0; i < 32; ++i) v[i] += r[i];
        }
        if (!last) {
          tmem_st32(trun + (uint32_t)c0, v);
        } else if (row < Mp) {
#pragma unroll
          for (int i = 0; i < 32; ++i)
            if (n0 + c0 + i < Np) Cs[(size_t)row * Np + n0 + c0 + i] = v[i];
        }
      }
      if (!last) {
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        mbar_arrive(acc_empty);
      }
    }
  }
  __syncwarp();
  const bool all_ok = __syncthreads_and(ok) != 0;
  if (!all_ok && tid == 0) atomicExch(err, 1);
  if (warp >= 2 && (nst == 0 || !all_ok)) {
    const int q = warp & 3;
    const int row = m0 + q * 32 + lane;
    float *Cs = C + ((size_t)prob * nsplit + split) * Mp * Np;
    if (row < Mp)
      for (int c = 0; c < kTcN; ++c)
        if (n0 + c < Np) Cs[(size_t)row * Np + n0 + c] = 0.0f;
  }
  if (tid == 0 && nst > 0 && !mbar_wait(done, 0)) atomicExch(err, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// rows x k (row-major FP64) -> rows x k4 FP32, zero padded to k4 columns
__global__ void pad_f32_kernel(const double *x, int rows, int k, int k4, float *y) {
  const long long n = (long long)rows * k4;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long r = i / k4, c = i % k4;
    y[i] = c < k ? (float)x[r * k + c] : 0.0f;
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

// 3D map over `batch` row-major [rows][Kp] FP32 matrices `sbatch` floats
// apart, box = 32 (K, 128 bytes) x box_rows x 1, 128-byte swizzle (the UMMA
// SWIZZLE_128B K-major layout).
static bool make_map(CUtensorMap *m, const float *ptr, int rows, int Kp, int box_rows, int batch,
                     long long sbatch) {
  auto fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)Kp, (cuuint64_t)rows, (cuuint64_t)batch};
  const cuuint64_t strides[2] = {(cuuint64_t)Kp * 4, (cuuint64_t)sbatch * 4};
  const cuuint32_t box[3] = {(cuuint32_t)kTcK, (cuuint32_t)box_rows, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)ptr, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

size_t tc_smem_bytes() { return (size_t)kStages * kStageBytes + 1024 + 256; }

int tc_tiles(int Mp, int Np) { return ((Mp + kTcM - 1) / kTcM) * ((Np + kTcN - 1) / kTcN); }

// Cpart[b][split][Mp][Np] = partial sums over K splits of A_b[Mp][Kp] .
// B_b[Np][Kp]^T for b < batch, split-TF32 tensor-core MMAs.  Operands FP32,
// 16-byte aligned, Kp % 4 == 0, batch strides sA, sB (floats, multiples of
// 4).  Returns the number of splits used in *used.
int tc_gemm_tf32x3_parts(const float *A, long long sA, const float *B, long long sB, int Mp, int Np, int Kp,
                         int batch, int splits, float *Cpart, int *d_err, int *used, cudaStream_t s) {
  if (Mp < 1 || Np < 1 || Kp < 4 || splits < 1 || batch < 1 || (Kp % 4)) return EMU_E_SHAPE;
  if (((uintptr_t)A & 15) || ((uintptr_t)B & 15) || (sA % 4) || (sB % 4)) return EMU_E_ARG;
  if (batch > 1 && (sA < (long long)Mp * Kp || sB < (long long)Np * Kp)) return EMU_E_ARG;
  TmaMaps maps;
  if (!make_map(&maps.a, A, Mp, Kp, kTcM, batch, batch > 1 ? sA : (long long)Mp * Kp) ||
      !make_map(&maps.b, B, Np, Kp, kTcN, batch, batch > 1 ? sB : (long long)Np * Kp))
    return EMU_E_CUDA;
  const size_t smem = tc_smem_bytes();
  if (cudaFuncSetAttribute(tc_tf32x3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return EMU_E_CUDA;
  int kper = (Kp + splits - 1) / splits;
  kper = (kper + kTcK - 1) / kTcK * kTcK;
  const int nsplit = (Kp + kper - 1) / kper;
  if ((long long)nsplit * batch > 65535) return EMU_E_SHAPE;
  dim3 grid((Np + kTcN - 1) / kTcN, (Mp + kTcM - 1) / kTcM, nsplit * batch);
  tc_tf32x3_kernel<<<grid, kTcThreads, smem, s>>>(maps, Mp, Np, Kp, kper, nsplit, Cpart, d_err);
  note_launch();
  *used = nsplit;
  return check_launch();
}

// C64[Mp][Np] = A[Mp][Kp] . B[Np][Kp]^T with split-TF32 tensor-core MMAs.
// Operands FP32 (16-byte aligned rows, Kp % 4 == 0); Cpart scratch
// [splits][Mp][Np] floats.
int tc_gemm_tf32x3(const float *A, const float *B, int Mp, int Np, int Kp, int splits, float *Cpart,
                   double *C64, int *d_err, cudaStream_t s) {
  int used = 0;
  const int st = tc_gemm_tf32x3_parts(A, (long long)Mp * Kp, B, (long long)Np * Kp, Mp, Np, Kp, 1, splits, Cpart,
                                      d_err, &used, s);
  if (st != EMU_OK) return st;
  const long long n = (long long)Mp * Np;
  int g = (int)((n + 255) / 256);
  if (g > 8 * sm_count()) g = 8 * sm_count();
  sum_splits_kernel<<<g, 256, 0, s>>>(Cpart, used, n, C64);
  note_launch(1);
  return check_launch();
}

}  // namespace emu

// Stand-alone entry for testing the tensor-core GEMM: C = A B^T (FP64 in,
// FP64 out, split-TF32 products with FP32 accumulation inside each split).
extern "C" size_t emu_tc_gemm_workspace_size(int m, int n, int k, int splits) {
  if (m < 1 || n < 1 || k < 1 || splits < 1) return 0;
  const size_t k4 = (size_t)(k + 3) / 4 * 4;
  const size_t a = (size_t)m * k4, b = (size_t)n * k4;
  return emu::align_up(4 * a, 256) + emu::align_up(4 * b, 256) +
         emu::align_up(4 * (size_t)splits * m * n, 256) + 256;
}

extern "C" int emu_tc_gemm_tf32x3(int m, int n, int k, const double *d_A, const double *d_B,
                                  double *d_C, int splits, int32_t *d_err, void *d_workspace,
                                  size_t workspace_bytes, void *stream) {
  if (m < 1 || n < 1 || k < 1 || splits < 1) return EMU_E_SHAPE;
  if (!d_A || !d_B || !d_C || !d_err) return EMU_E_ARG;
  if (!d_workspace || workspace_bytes < emu_tc_gemm_workspace_size(m, n, k, splits)) return EMU_E_WORKSPACE;
  if ((uintptr_t)d_workspace & 255) return EMU_E_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int k4 = (k + 3) / 4 * 4;
  const size_t a = (size_t)m * k4, b = (size_t)n * k4;
  char *w = (char *)d_workspace;
  float *A32 = (float *)w;
  float *B32 = (float *)(w + emu::align_up(4 * a, 256));
  float *Cp = (float *)(w + emu::align_up(4 * a, 256) + emu::align_up(4 * b, 256));
  const int sms = emu::sm_count();
  pad_f32_kernel<<<8 * sms, 256, 0, s>>>(d_A, m, k, k4, A32);
  pad_f32_kernel<<<8 * sms, 256, 0, s>>>(d_B, n, k, k4, B32);
  emu::note_launch(2);
  return emu::tc_gemm_tf32x3(A32, B32, m, n, k4, splits, Cp, d_C, (int *)d_err, s);
}
