// FP64 FMA throughput probe: the denominator of the FP64 roofline of the
// film kernels (the driver-measured peaks cover HBM copy and bf16 GEMM only).
#include <cuda_runtime.h>

#include "emu_internal.h"

namespace {

__global__ void __launch_bounds__(256) dfma_probe(int iters, double seed, double *out) {
  double a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3;
  double a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
  const double m = 0.999999, c = 1e-7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
      a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
    }
  }
  const double s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == 12345.678) out[blockIdx.x] = s;  // keeps the chains live
}

}  // namespace

// FLOPs performed = 2 * 64 * iters * threads * blocks.
extern "C" int emu_probe_fp64(int blocks, int threads, int iters, double *d_out, void *stream) {
  if (blocks < 1 || threads < 1 || threads > 256 || iters < 1 || !d_out) return EMU_E_ARG;
  dfma_probe<<<blocks, threads, 0, (cudaStream_t)stream>>>(iters, 1.0, d_out);
  emu::note_launch();
  return emu::check_launch();
}
