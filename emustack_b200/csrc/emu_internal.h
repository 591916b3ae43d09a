// Internal helpers shared by the translation units of libemustack_gsm.so.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/emustack_gsm.h"

namespace emu {

// Counts kernel launches made by this library (reported by emu_launch_count).
void note_launch(int n = 1);

// Map the last CUDA error to a status (and clear it).
inline int cuda_status(cudaError_t e) { return e == cudaSuccess ? EMU_OK : EMU_E_CUDA; }

inline int check_launch() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? EMU_OK : EMU_E_CUDA;
}

// Number of SMs of the current device (cached per device).
int sm_count();

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Tensor-core split-TF32 GEMM (tc_gemm.cu): C64[Mp][Np] = A[Mp][Kp] . B[Np][Kp]^T
// from FP32 operands (split into TF32 hi/lo inside the kernel); Cpart is
// scratch of splits * Mp * Np floats.
int tc_gemm_tf32x3(const float *A, const float *B, int Mp, int Np, int Kp, int splits, float *Cpart,
                   double *C64, int *d_err, cudaStream_t s);
// Batched form: Cpart[b][split][Mp][Np] partial sums for b < batch (operand
// batch strides sA, sB in floats); *used = number of K splits taken.
int tc_gemm_tf32x3_parts(const float *A, long long sA, const float *B, long long sB, int Mp, int Np, int Kp,
                         int batch, int splits, float *Cpart, int *d_err, int *used, cudaStream_t s);
// output tiles of one K split
int tc_tiles(int Mp, int Np);


// process-wide choice for the dense interface / cascade paths (0 automatic,
// 1 one CTA per problem, 2 multi-CTA), set by emu_set_dense_mode
int dense_mode();
size_t tc_smem_bytes();

}  // namespace emu
