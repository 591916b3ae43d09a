// Fused all-film GSM kernel: k_z, sort order, impedances, Fresnel interfaces,
// cascade and energy fluxes for a batch of spectral points in one launch.
//
// When every layer of a stack is a homogeneous film (reference: Anallo),
// every matrix of backend/stack.py:162-426 is diagonal, so the reference's
// dense solves and products collapse to independent scalar recursions, one
// per plane-wave order and polarisation.  The reference still runs them as
// dense P x P LAPACK solves; here each order is one thread.
//
// Mapping: a CTA of 256 threads holds `ppc` points at a time, a team of
// `team` threads per point, one thread per order (looping when Npw > team).
// Both polarisations of an order share one thread (they share k_z).
//
// Phases per CTA iteration (all threads take every __syncthreads):
//   0  per-point constants in shared memory: each layer's n, k = 2 pi n / wl,
//      1/n, 1/k and the heights
//   1  air k_z with the Wood-anomaly check (backend/mode_calcs.py:147-162),
//      sort keys -Re k_z + Im k_z (backend/mode_calcs.py:164-171) and the
//      air's propagating-order count
//   2  (only if the air hit a Wood anomaly) air k_z again with k_parallel
//      scaled by 1 - 1e-9
//   3  rank of each order = its position in the sorted order (stable on
//      ties; ties only occur at exactly degenerate orders, whose values are
//      identical), specular order = rank of (0, 0), propagating counts of
//      substrate and superstrate
//   4  Wood check of every layer (k^2 - alpha^2 - beta^2 == 0), then per
//      order: bottom-to-top cascade for both polarisations (R_net, T_net)
//      and, for the order(s) that carry incident light, the top-to-bottom
//      flux pass over the scalars saved in the workspace, summed per level
//      in shared memory
//   5  (only if a layer hit a Wood anomaly) phase 4 again for those points
//      with k_parallel scaled by 1 - 1e-9 in the marked layers
//   6  a_list / t_list / r_list (backend/stack.py:368-426)
// Divisions use the Newton reciprocal of emu_fastmath.cuh.  The decisions
// taken on k_z (exact zeros at Wood anomalies, exactly real k_z of
// propagating orders, the sort keys) use IEEE square roots and quotients;
// the k_z entering the recursion comes from the Newton form, which is exactly
// zero, real or imaginary for the same arguments.
#include <cuda_runtime.h>

#include "emu_cplx.cuh"
#include "emu_fastmath.cuh"
#include "emu_internal.h"
#include "emu_modes.cuh"
#include "film_core.cuh"

namespace {

using namespace emu;

// Launch variants (EmuFilmStackBatch.variant): threads per CTA and the
// minimum resident CTAs per SM given to the compiler (which sets the
// register cap: 65536 / (threads * min CTAs), at most 255).
constexpr int kVariants = 6;
constexpr int kMaxCtaSmem = 200 * 1024;
constexpr int kVarThreadsTab[kVariants] = {256, 128, 512, 256, 256, 256};

struct FilmArgs {
  EmuFilmStackBatch p;
  int team;        // threads per point
  int ppc;         // points per CTA iteration
  int n_act;       // active-order slots per point in the workspace
  cd *ws;          // [B][n_act][L][2][kSave]
  double dy;       // period_y / period
  double inv_sqrt2;
};

// Point accessor over the uniform batch: every field is derived from the
// kernel parameters and the point index when used.  kPlain: the request asks
// for no optional output, has no shears and a standard polarisation, so
// those accessors are compile-time NULL and the recursion carries none of
// their checks or live values.
template <bool kPlain>
struct UniformPoint {
  const FilmArgs &a;
  int b;
  __device__ int L() const { return a.p.n_layers; }
  __device__ int npw() const { return a.p.n_pw; }
  __device__ int P() const { return 2 * a.p.n_pw; }
  __device__ int world_1d() const { return a.p.world_1d; }
  __device__ int pol() const { return a.p.pol; }
  __device__ int ncoord() const { return a.p.shear_ncoord; }
  __device__ bool slot_per_order() const { return !kPlain && a.p.pol == EMU_POL_INCOMING; }
  __device__ double dy() const { return a.dy; }
  __device__ double period() const { return a.p.period; }
  __device__ double inv_sqrt2() const { return a.inv_sqrt2; }
  __device__ const int32_t *px() const { return a.p.d_px; }
  __device__ const int32_t *py() const { return a.p.d_py; }
  __device__ const emu_c128 *incoming() const { return a.p.d_incoming + (size_t)b * P(); }
  __device__ const double *shears() const { return kPlain ? nullptr : a.p.d_shears; }
  __device__ cd *ws() const { return a.ws + (size_t)b * a.n_act * L() * 2 * kSave; }
  __device__ emu_c128 *R_net() const { return a.p.d_R_net + (size_t)b * P(); }
  __device__ emu_c128 *T_net() const { return a.p.d_T_net + (size_t)b * P(); }
  __device__ emu_c128 *kz() const {
    return (!kPlain && a.p.d_kz) ? a.p.d_kz + (size_t)b * L() * npw() : nullptr;
  }
  __device__ emu_c128 *layer_rt() const {
    return (!kPlain && a.p.d_layer_rt) ? a.p.d_layer_rt + (size_t)b * L() * 2 * P() : nullptr;
  }
  __device__ emu_c128 *vcd() const {
    return (!kPlain && a.p.d_vec_coef_down) ? a.p.d_vec_coef_down + (size_t)b * L() * P() : nullptr;
  }
  __device__ emu_c128 *vcu() const {
    return (!kPlain && a.p.d_vec_coef_up) ? a.p.d_vec_coef_up + (size_t)b * (L() - 1) * P()
                                           : nullptr;
  }
  __device__ double wl_nm() const { return a.p.d_wl_nm[b]; }
  __device__ double kx() const { return a.p.d_k_pll[2 * (size_t)b]; }
  __device__ double ky() const { return a.p.d_k_pll[2 * (size_t)b + 1]; }
  __device__ emu_c128 n(int i) const { return a.p.d_n[(size_t)b * L() + i]; }
  __device__ double height(int i) const {
    return a.p.d_heights_nm[(a.p.heights_per_point ? (size_t)b * (L() - 2) : 0) + i];
  }
  __device__ int32_t *sort_order() const {
    return (!kPlain && a.p.d_sort_order) ? a.p.d_sort_order + (size_t)b * npw() : nullptr;
  }
  __device__ int32_t *specular() const {
    return (!kPlain && a.p.d_specular) ? a.p.d_specular + b : nullptr;
  }
  __device__ int32_t *num_prop() const {
    return (!kPlain && a.p.d_num_prop) ? a.p.d_num_prop + (size_t)b * (L() + 1) : nullptr;
  }
  __device__ double *fluxes() const {
    return (!kPlain && a.p.d_fluxes) ? a.p.d_fluxes + (size_t)b * (L() + 1) * 2 : nullptr;
  }
  __device__ double *a_list() const { return a.p.d_a_list + (size_t)b * (L() - 1); }
  __device__ double *t_list() const { return a.p.d_t_list + (size_t)b * (L() - 1); }
  __device__ double *r_list() const { return a.p.d_r_list + b; }
  __device__ uint32_t *flags() const { return a.p.d_flags + b; }
};

template <int kThreads, int kMinBlocks, bool kPlain>
__global__ void __launch_bounds__(kThreads, kMinBlocks) film_stack_kernel(FilmArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const EmuFilmStackBatch &p = a.p;
  const int B = p.n_points;
  const int team = a.team, ppc = a.ppc;
  const int slot = threadIdx.x / team;
  const bool in_slot = slot < ppc;
  const SlotSmem S = slot_layout(p.n_pw, p.n_layers, p.pol != EMU_POL_INCOMING);
  unsigned char *base = smem + (in_slot ? slot : 0) * S.stride;
  const CtaTeam tm{(int)(threadIdx.x % team), team};
  for (int bb = blockIdx.x * ppc; bb < B; bb += gridDim.x * ppc) {
    const int b = bb + slot;
    film_point(tm, UniformPoint<kPlain>{a, b}, in_slot && b < B, base, S);
  }
}

struct Launch {
  int team, ppc, n_act;
  size_t smem;
};

using FilmKernel = void (*)(FilmArgs);
// 0: 256 threads x 2 CTAs (128 registers), 1: 128 x 4 (128), 2: 512 x 1
// (128), 3: 256 x 1 (255 registers, no spills, half the resident warps),
// 4: 256 x 3 (85 registers), 5: 256 x 4 (64): more warps to hide the FP64
// latency chains, at the price of spills to L1.  Row 1: the plain
// specialisation (see UniformPoint), same arithmetic, same results.
const FilmKernel kVarKernels[2][kVariants] = {
    {film_stack_kernel<256, 2, false>, film_stack_kernel<128, 4, false>,
     film_stack_kernel<512, 1, false>, film_stack_kernel<256, 1, false>,
     film_stack_kernel<256, 3, false>, film_stack_kernel<256, 4, false>},
    {film_stack_kernel<256, 2, true>, film_stack_kernel<128, 4, true>,
     film_stack_kernel<512, 1, true>, film_stack_kernel<256, 1, true>,
     film_stack_kernel<256, 3, true>, film_stack_kernel<256, 4, true>}};

// True when the request needs none of what the plain specialisation drops.
bool is_plain(const EmuFilmStackBatch *p) {
  return p->pol != EMU_POL_INCOMING && !p->d_shears && !p->d_kz && !p->d_layer_rt &&
         !p->d_vec_coef_down && !p->d_vec_coef_up && !p->d_fluxes && !p->d_sort_order &&
         !p->d_specular && !p->d_num_prop;
}

Launch plan(const EmuFilmStackBatch *p) {
  Launch l;
  const int threads = kVarThreadsTab[p->variant];
  l.team = p->n_pw <= threads ? p->n_pw : threads;
  l.ppc = threads / l.team;
  // at most kMaxCtaSmem of slots per CTA (small order sets, many points)
  const int stride = slot_layout(p->n_pw, p->n_layers, p->pol != EMU_POL_INCOMING).stride;
  if (l.ppc * stride > kMaxCtaSmem) l.ppc = kMaxCtaSmem / stride > 0 ? kMaxCtaSmem / stride : 1;
  l.n_act = (p->pol == EMU_POL_INCOMING) ? p->n_pw : 1;
  l.smem = (size_t)stride * l.ppc;
  return l;
}

int validate(const EmuFilmStackBatch *p) {
  if (!p) return EMU_E_ARG;
  if (p->n_points < 0 || p->n_layers < 2 || p->n_pw < 1) return EMU_E_SHAPE;
  if (!(p->period > 0) || !(p->period_y > 0)) return EMU_E_ARG;
  if (p->pol < EMU_POL_INCOMING || p->pol > EMU_POL_LCIRC) return EMU_E_ARG;
  if (p->pol == EMU_POL_INCOMING && !p->d_incoming) return EMU_E_ARG;
  if (p->n_points > 0 &&
      (!p->d_px || !p->d_py || !p->d_wl_nm || !p->d_k_pll || !p->d_n || !p->d_R_net ||
       !p->d_T_net || !p->d_a_list || !p->d_t_list || !p->d_r_list || !p->d_flags))
    return EMU_E_ARG;
  if (p->n_layers > 2 && p->n_points > 0 && !p->d_heights_nm) return EMU_E_ARG;
  if ((p->d_vec_coef_down == nullptr) != (p->d_vec_coef_up == nullptr)) return EMU_E_ARG;
  if (p->d_shears && p->shear_ncoord != 1 && p->shear_ncoord != 2) return EMU_E_ARG;
  if (p->variant < 0 || p->variant >= kVariants) return EMU_E_ARG;
  if (slot_layout(p->n_pw, p->n_layers, p->pol != EMU_POL_INCOMING).stride > kMaxCtaSmem) return EMU_E_SHAPE;
  return EMU_OK;
}

}  // namespace

// Only incoming amplitudes use the global workspace (any order may carry
// light, so each order keeps its flux-pass scalars there); every other
// polarisation keeps them in shared memory and needs no workspace.
extern "C" size_t emu_film_stack_workspace_size(const EmuFilmStackBatch *p) {
  if (validate(p) != EMU_OK) return 0;
  if (p->pol != EMU_POL_INCOMING) return 0;
  const Launch l = plan(p);
  return (size_t)p->n_points * l.n_act * p->n_layers * 2 * kSave * sizeof(cd);
}

extern "C" int emu_film_stack_batch(const EmuFilmStackBatch *p, void *d_workspace,
                                    size_t workspace_bytes, void *stream) {
  int st = validate(p);
  if (st != EMU_OK) return st;
  if (p->n_points == 0) return EMU_OK;
  const size_t need = emu_film_stack_workspace_size(p);
  if (need > 0 && (!d_workspace || workspace_bytes < need)) return EMU_E_WORKSPACE;
  const Launch l = plan(p);
  FilmArgs a;
  a.p = *p;
  a.team = l.team;
  a.ppc = l.ppc;
  a.n_act = l.n_act;
  a.ws = (cd *)d_workspace;
  a.dy = p->period_y / p->period;
  a.inv_sqrt2 = 1.0 / sqrt(2.0);
  const FilmKernel kern = kVarKernels[is_plain(p) ? 1 : 0][p->variant];
  const int threads = kVarThreadsTab[p->variant];
  if (l.smem > 48 * 1024) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)l.smem) !=
        cudaSuccess)
      return EMU_E_CUDA;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, l.smem) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const long long groups = ((long long)p->n_points + l.ppc - 1) / l.ppc;
  long long grid = (long long)emu::sm_count() * per_sm;
  if (grid > groups) grid = groups;
  kern<<<(int)grid, threads, l.smem, (cudaStream_t)stream>>>(a);
  emu::note_launch();
  return emu::check_launch();
}

// ---------------------------------------------------------------------------
// Allocation-free entry point.
//
// Some callers cannot allocate device memory at the point where they solve:
// a host thread inside a latency-critical loop (cudaMalloc and cudaFree
// synchronise the device), code that runs while another framework owns the
// device heap through its own caching allocator, or an embedding that must
// not fail on memory pressure after start-up.  For them the film solve can
// use a fixed scratch array compiled into this library instead of a
// caller-provided workspace.  The array lives in every GPU that loads the
// library, for the life of the process.
#include <mutex>

namespace {

constexpr size_t kStaticScratchBytes = (size_t)16 << 20;  // 16 MiB
static __device__ __align__(256) unsigned char g_film_scratch[kStaticScratchBytes];

std::mutex g_scratch_mu;
void *g_scratch_addr[64] = {nullptr};

}  // namespace

extern "C" size_t emu_film_stack_static_scratch_bytes(void) { return kStaticScratchBytes; }

extern "C" int emu_film_stack_batch_noalloc(const EmuFilmStackBatch *p, void *stream) {
  int st = validate(p);
  if (st != EMU_OK) return st;
  if (p->n_points == 0) return EMU_OK;
  if (emu_film_stack_workspace_size(p) > kStaticScratchBytes) return EMU_E_WORKSPACE;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return EMU_E_CUDA;
  void *addr = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
      // the host-side name of the array is not a device address: ask the
      // runtime for this device's copy once, with the device current
      if (cudaGetSymbolAddress(&g_scratch_addr[dev], g_film_scratch) != cudaSuccess) {
        g_scratch_addr[dev] = nullptr;
        cudaGetLastError();
        return EMU_E_CUDA;
      }
    }
    addr = g_scratch_addr[dev];
  }
  return emu_film_stack_batch(p, addr, kStaticScratchBytes, stream);
}
