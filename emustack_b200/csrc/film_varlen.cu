// All-film GSM solve for batches of points with different shapes: one warp
// per point, any mix of layer counts, order sets, periods, polarisations,
// wavelengths and k_parallel in one launch.
//
// The reference solves each of these with its own Stack(layers).calc_scat
// call (backend/stack.py:162-426), looping over wavelengths or spreading them
// over a process pool.  Here a point is a descriptor (EmuFilmPoint) with
// offsets into packed per-point arrays; a warp reads its descriptor, runs
// the same phases as the uniform kernel of film_stack.cu (film_core.cuh,
// with warp barriers in place of CTA barriers) and writes its outputs at
// offsets the host plan assigned.
//
// Layout: a CTA of `warps` warps owns warps * slot bytes of shared memory,
// one slot per warp sized for the batch's largest (Npw, L).  Points are
// visited in the plan's costliest-first order (Npw * L descending), so the
// long points start first and the grid-stride tail is made of short ones.
#include <cuda_runtime.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "emu_cplx.cuh"
#include "emu_fastmath.cuh"
#include "emu_internal.h"
#include "emu_modes.cuh"
#include "film_core.cuh"

namespace {

using namespace emu;

constexpr int kVarThreads = 256;
constexpr int kMaxSlotBytes = 200 * 1024;

struct VarArgs {
  EmuFilmVarBatch p;
  const EmuFilmPoint *pts;
  unsigned char *ws;
  int64_t ws_bytes;
  double inv_sqrt2_;
  int warps;  // warps per CTA actually used
};

// Point accessor over one descriptor; the scalars used in the inner loops
// are held in registers, the offsets are read from the descriptor on use.
struct VarPoint {
  const VarArgs &a;
  const EmuFilmPoint *d;
  int b, L_, npw_, w1d_, pol_;
  double dy_, period_;
  __device__ int L() const { return L_; }
  __device__ int npw() const { return npw_; }
  __device__ int world_1d() const { return w1d_; }
  __device__ int pol() const { return pol_; }
  __device__ int ncoord() const { return 1; }
  __device__ bool slot_per_order() const { return pol_ == EMU_POL_INCOMING; }
  __device__ double dy() const { return dy_; }
  __device__ double period() const { return period_; }
  __device__ double inv_sqrt2() const { return a.inv_sqrt2_; }
  __device__ const int32_t *px() const { return a.p.d_px + d->order_off; }
  __device__ const int32_t *py() const { return a.p.d_py + d->order_off; }
  __device__ const emu_c128 *incoming() const { return a.p.d_incoming + d->inc_off; }
  __device__ const double *shears() const { return nullptr; }
  __device__ cd *ws() const { return (cd *)(a.ws + d->ws_off); }
  __device__ emu_c128 *R_net() const { return a.p.d_R_net + d->rt_off; }
  __device__ emu_c128 *T_net() const { return a.p.d_T_net + d->rt_off; }
  __device__ emu_c128 *kz() const { return nullptr; }
  __device__ emu_c128 *layer_rt() const { return nullptr; }
  __device__ emu_c128 *vcd() const { return nullptr; }
  __device__ emu_c128 *vcu() const { return nullptr; }
  __device__ double wl_nm() const { return d->wl_nm; }
  __device__ double kx() const { return d->kx; }
  __device__ double ky() const { return d->ky; }
  __device__ emu_c128 n(int i) const { return a.p.d_n[d->n_off + i]; }
  __device__ double height(int i) const { return a.p.d_heights_nm[d->h_off + i]; }
  __device__ int32_t *sort_order() const { return nullptr; }
  __device__ int32_t *specular() const { return a.p.d_specular ? a.p.d_specular + b : nullptr; }
  __device__ int32_t *num_prop() const {
    return a.p.d_num_prop ? a.p.d_num_prop + d->np_off : nullptr;
  }
  __device__ double *fluxes() const { return nullptr; }
  __device__ double *a_list() const { return a.p.d_a_list + d->list_off; }
  __device__ double *t_list() const { return a.p.d_t_list + d->list_off; }
  __device__ double *r_list() const { return a.p.d_r_list + b; }
  __device__ uint32_t *flags() const { return a.p.d_flags + b; }
};

__host__ __device__ inline int64_t ws_bytes_of(int L, int npw, int pol) {
  const int64_t n_act = pol == EMU_POL_INCOMING ? npw : 1;
  return n_act * L * 2 * kSave * (int64_t)sizeof(cd);
}

// [off, off + len) inside [0, cap)
__device__ __forceinline__ bool inside(int64_t off, int64_t len, int64_t cap) {
  return off >= 0 && len >= 0 && off <= cap && len <= cap - off;
}

__device__ __forceinline__ bool point_ok(const VarArgs &a, const EmuFilmPoint *d) {
  const EmuFilmVarBatch &p = a.p;
  const int L = d->n_layers, npw = d->n_pw, pol = d->pol;
  if (L < 2 || L > p.max_layers || npw < 1 || npw > p.max_pw) return false;
  if (pol < EMU_POL_INCOMING || pol > EMU_POL_LCIRC) return false;
  if (!(d->period > 0) || !(d->period_y > 0)) return false;
  if (!inside(d->order_off, npw, p.order_len) || !inside(d->n_off, L, p.n_len) ||
      !inside(d->rt_off, 2 * npw, p.rt_len) || !inside(d->list_off, L - 1, p.list_len))
    return false;
  if (L > 2 && (!p.d_heights_nm || !inside(d->h_off, L - 2, p.h_len))) return false;
  if (pol == EMU_POL_INCOMING && (!p.d_incoming || !inside(d->inc_off, 2 * npw, p.inc_len)))
    return false;
  if (p.d_num_prop && !inside(d->np_off, L + 1, p.np_len)) return false;
  if ((d->ws_off & 15) != 0 || !inside(d->ws_off, ws_bytes_of(L, npw, pol), a.ws_bytes))
    return false;
  return true;
}

// kMinBlocks: CTAs per SM the register budget is cut for (2: 128 registers;
// 3: 85, more resident warps, some values spilled to L1).
template <int kMinBlocks>
__global__ void __launch_bounds__(kVarThreads, kMinBlocks) film_var_kernel(VarArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp >= a.warps) return;  // whole warps leave; no CTA barrier follows
  const SlotSmem S = slot_layout(a.p.max_pw, a.p.max_layers);
  unsigned char *base = smem + warp * S.stride;
  const WarpTeam tm{lane};
  const int B = a.p.n_points;
  for (int w = blockIdx.x * a.warps + warp; w < B; w += gridDim.x * a.warps) {
    const int b = a.p.d_order ? a.p.d_order[w] : w;
    if (b < 0 || b >= B) continue;  // warp-uniform
    const EmuFilmPoint *d = a.pts + b;
    if (!point_ok(a, d)) {
      if (lane == 0) a.p.d_flags[b] = EMU_PT_BAD_POINT;
      continue;
    }
    const VarPoint pt{a,         d,           b,        d->n_layers, d->n_pw, d->world_1d,
                      d->pol,    d->period_y / d->period, d->period};
    film_point(tm, pt, true, base, S);
  }
}

}  // namespace

extern "C" int emu_film_var_plan(EmuFilmPoint *h, int n, int32_t *h_order, int64_t *rt_len,
                                 int64_t *list_len, int64_t *np_len, size_t *workspace_bytes,
                                 int *max_layers, int *max_pw) {
  if (n < 0 || (n > 0 && !h)) return EMU_E_ARG;
  int64_t rt = 0, li = 0, np = 0, ws = 0;
  int ml = 2, mp = 1;
  for (int i = 0; i < n; ++i) {
    EmuFilmPoint &q = h[i];
    if (q.n_layers < 2 || q.n_pw < 1) return EMU_E_SHAPE;
    if (q.pol < EMU_POL_INCOMING || q.pol > EMU_POL_LCIRC) return EMU_E_ARG;
    if (!(q.period > 0) || !(q.period_y > 0)) return EMU_E_ARG;
    q.rt_off = rt;
    rt += 2 * (int64_t)q.n_pw;
    q.list_off = li;
    li += q.n_layers - 1;
    q.np_off = np;
    np += q.n_layers + 1;
    q.ws_off = ws;
    ws += (int64_t)align_up((size_t)ws_bytes_of(q.n_layers, q.n_pw, q.pol), 16);
    ml = std::max(ml, (int)q.n_layers);
    mp = std::max(mp, (int)q.n_pw);
  }
  if (slot_layout(mp, ml).stride > kMaxSlotBytes) return EMU_E_SHAPE;
  if (h_order) {
    std::vector<int32_t> ord(n);
    std::iota(ord.begin(), ord.end(), 0);
    // costliest first: rank computation O(Npw^2), cascade O(Npw L)
    auto cost = [&](int i) {
      const int64_t m = h[i].n_pw;
      return m * m + 8 * m * h[i].n_layers;
    };
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return cost(x) > cost(y); });
    std::copy(ord.begin(), ord.end(), h_order);
  }
  if (rt_len) *rt_len = rt;
  if (list_len) *list_len = li;
  if (np_len) *np_len = np;
  if (workspace_bytes) *workspace_bytes = (size_t)ws;
  if (max_layers) *max_layers = ml;
  if (max_pw) *max_pw = mp;
  return EMU_OK;
}

extern "C" int emu_film_var_batch(const EmuFilmVarBatch *p, void *d_workspace,
                                  size_t workspace_bytes, void *stream) {
  if (!p) return EMU_E_ARG;
  if (p->n_points < 0 || p->max_layers < 2 || p->max_pw < 1) return EMU_E_SHAPE;
  if (p->n_points == 0) return EMU_OK;
  if (!p->d_points || !p->d_px || !p->d_py || !p->d_n || !p->d_R_net || !p->d_T_net ||
      !p->d_a_list || !p->d_t_list || !p->d_r_list || !p->d_flags)
    return EMU_E_ARG;
  if (!d_workspace) return EMU_E_WORKSPACE;
  const int stride = slot_layout(p->max_pw, p->max_layers).stride;
  if (stride > kMaxSlotBytes) return EMU_E_SHAPE;
  VarArgs a;
  a.p = *p;
  a.pts = p->d_points;
  a.ws = (unsigned char *)d_workspace;
  a.ws_bytes = (int64_t)workspace_bytes;
  a.inv_sqrt2_ = 1.0 / sqrt(2.0);
  if (p->warps_per_cta < 0 || p->warps_per_cta > kVarThreads / 32) return EMU_E_ARG;
  if (p->variant < 0 || p->variant > 1) return EMU_E_ARG;
  const auto kern = p->variant ? film_var_kernel<3> : film_var_kernel<2>;
  a.warps = std::max(1, std::min(kVarThreads / 32, kMaxSlotBytes / stride));
  if (p->warps_per_cta > 0) a.warps = std::min(a.warps, p->warps_per_cta);
  const size_t smem = (size_t)stride * a.warps;
  if (smem > 48 * 1024) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
      return EMU_E_CUDA;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * a.warps, smem) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const long long groups = ((long long)p->n_points + a.warps - 1) / a.warps;
  long long grid = (long long)emu::sm_count() * per_sm;
  if (grid > groups) grid = groups;
  kern<<<(int)grid, 32 * a.warps, smem, (cudaStream_t)stream>>>(a);
  emu::note_launch();
  return emu::check_launch();
}
