// Device-resident request loop for all-film GSM solves.
//
// A persistent kernel serves spectral-point requests that the host writes
// into a ring of slots in pinned, device-mapped host memory: the host never
// launches a kernel per request or per batch.  Each request is one
// Stack(layers).calc_scat(pol) of an all-film stack (backend/stack.py:
// 162-426) with its own layer count, order set, periods, polarisation,
// wavelength and k_parallel; the kernel's warps solve requests as they
// arrive, one warp per request, with the film recursion of film_core.cuh,
// and write R_net / T_net diagonals, a_list, t_list, r_list and flags back
// into the request's slot, then its completion word.
//
// Protocol (memory in the ring's control block and slots is host memory):
//   host  : writes the request into slot ticket % capacity, a release
//           fence, then tail = ticket + 1;
//   device: one doorbell lane (block 0, warp 0) polls tail with system-scope
//           acquire loads and publishes it to a device-memory mirror; the
//           other warps claim tickets below the mirror by compare-and-swap on
//           a device counter, copy the slot's inputs to device memory (loads
//           that bypass the caches), solve, copy the outputs into the slot,
//           fence at system scope and store done = ticket + 1;
//   host  : polls done, an acquire fence, reads the outputs.
// A slot is reused only after the host has read its previous result.
//
// Every wait is bounded.  The doorbell ends the loop when no request has
// arrived for idle_seconds (and all are claimed) or when the host sets
// stop; before it ends on idle it marks the control block `exited` and
// re-reads tail once, so a request submitted at that moment either keeps the
// loop alive or finds `exited` set and restarts it (the host writes tail
// before it reads `exited`, the device writes `exited` before it re-reads
// tail, both with full fences between).  Workers leave when the doorbell
// has ended the loop and nothing is left to claim, or after a poll limit
// far above the idle time (then status EMU_E_TIMEOUT).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "emu_cplx.cuh"
#include "emu_fastmath.cuh"
#include "emu_internal.h"
#include "emu_modes.cuh"
#include "film_core.cuh"

namespace {

using namespace emu;

constexpr int kRingNpw = EMU_RING_MAX_PW;   // orders per polarisation
constexpr int kRingL = EMU_RING_MAX_LAYERS;  // layers incl. substrate, superstrate
constexpr int kRingWarps = 8;               // warps per CTA
constexpr int kRingThreads = 32 * kRingWarps;

// ---- slot layout (bytes; every block 16-byte aligned)
struct SlotHdr {
  int32_t n_layers, n_pw, world_1d, pol;
  double period, period_y, wl_nm, kx, ky;
  double pad;
};
static_assert(sizeof(SlotHdr) == 64, "slot header");
constexpr size_t kOffHdr = 0;
constexpr size_t kOffPx = kOffHdr + sizeof(SlotHdr);
constexpr size_t kOffPy = kOffPx + 4 * kRingNpw;
constexpr size_t kOffN = kOffPy + 4 * kRingNpw;
constexpr size_t kOffH = kOffN + 16 * kRingL;
constexpr size_t kInBytes = kOffH + 8 * kRingL;  // inputs: [0, kInBytes)
constexpr size_t kOffDone = kInBytes;             // int64 done, uint32 flags, int32 status
constexpr size_t kOffOut = kOffDone + 16;         // outputs copied as one block
constexpr size_t kOffR = kOffOut;
constexpr size_t kOffT = kOffR + 16 * 2 * kRingNpw;
constexpr size_t kOffA = kOffT + 16 * 2 * kRingNpw;
constexpr size_t kOffTl = kOffA + 8 * kRingL;
constexpr size_t kOffRl = kOffTl + 8 * kRingL;
constexpr size_t kOffFl = kOffRl + 8;
constexpr size_t kOutBytes = (kOffFl + 8) - kOffOut;
constexpr size_t kSlotBytes = (kOffOut + kOutBytes + 255) / 256 * 256;
static_assert(kInBytes % 16 == 0 && kOutBytes % 16 == 0 && (kOffFl + 8 - kOffA) % 16 == 0 &&
                  kOffPx % 16 == 0 && kOffPy % 16 == 0 && kOffN % 16 == 0 && kOffH % 16 == 0,
              "16-byte blocks");
// per-warp device staging: the inputs, then the outputs, same offsets
constexpr size_t kStageBytes = kSlotBytes;

struct RingCtl {
  int64_t tail;    // host: requests submitted
  int32_t stop;    // host: 1 ends the loop
  int32_t exited;  // device: the loop decided to end
  int32_t status;  // device: EMU_OK or EMU_E_TIMEOUT
  int32_t pad[59];
};
static_assert(sizeof(RingCtl) == 256, "control block");

struct RingDev {
  unsigned long long head;  // next ticket to claim
  unsigned long long tail;  // mirror of the host's tail
  int stop;                 // 0 run, 1 host stop, 2 idle end
  int pad[3];
};

struct RingArgs {
  RingCtl *ctl;           // device view of the mapped control block
  unsigned char *slots;   // device view of the mapped slots
  long long cap;
  RingDev *dev;
  unsigned char *stage;   // [warps][kStageBytes]
  unsigned long long idle_ns;
  unsigned sleep_ns;
  double inv_sqrt2;
};

// ---- memory-model helpers
__device__ __forceinline__ long long ld_acquire_sys(const int64_t *p) {
  long long v;
  asm volatile("ld.acquire.sys.global.s64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_volatile_i32(const int32_t *p) {
  return *(const volatile int32_t *)p;
}
__device__ __forceinline__ unsigned long long ld_acquire_gpu(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned long long *p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Point accessor over a staged request.
struct RingPoint {
  const SlotHdr *h;
  unsigned char *st;
  double inv_sqrt2_, dy_;
  __device__ int L() const { return h->n_layers; }
  __device__ int npw() const { return h->n_pw; }
  __device__ int world_1d() const { return h->world_1d; }
  __device__ int pol() const { return h->pol; }
  __device__ int ncoord() const { return 1; }
  __device__ bool slot_per_order() const { return false; }
  __device__ double dy() const { return dy_; }
  __device__ double period() const { return h->period; }
  __device__ double inv_sqrt2() const { return inv_sqrt2_; }
  __device__ const int32_t *px() const { return (const int32_t *)(st + kOffPx); }
  __device__ const int32_t *py() const { return (const int32_t *)(st + kOffPy); }
  __device__ const emu_c128 *incoming() const { return nullptr; }
  __device__ const double *shears() const { return nullptr; }
  __device__ cd *ws() const { return nullptr; }
  __device__ emu_c128 *R_net() const { return (emu_c128 *)(st + kOffR); }
  __device__ emu_c128 *T_net() const { return (emu_c128 *)(st + kOffT); }
  __device__ emu_c128 *kz() const { return nullptr; }
  __device__ emu_c128 *layer_rt() const { return nullptr; }
  __device__ emu_c128 *vcd() const { return nullptr; }
  __device__ emu_c128 *vcu() const { return nullptr; }
  __device__ double wl_nm() const { return h->wl_nm; }
  __device__ double kx() const { return h->kx; }
  __device__ double ky() const { return h->ky; }
  __device__ emu_c128 n(int i) const { return ((const emu_c128 *)(st + kOffN))[i]; }
  __device__ double height(int i) const { return ((const double *)(st + kOffH))[i]; }
  __device__ int32_t *sort_order() const { return nullptr; }
  __device__ int32_t *specular() const { return nullptr; }
  __device__ int32_t *num_prop() const { return nullptr; }
  __device__ double *fluxes() const { return nullptr; }
  __device__ double *a_list() const { return (double *)(st + kOffA); }
  __device__ double *t_list() const { return (double *)(st + kOffTl); }
  __device__ double *r_list() const { return (double *)(st + kOffRl); }
  __device__ uint32_t *flags() const { return (uint32_t *)(st + kOffFl); }
};

__device__ __forceinline__ bool request_ok(const SlotHdr *h) {
  const int L = h->n_layers, npw = h->n_pw, pol = h->pol;
  return L >= 2 && L <= kRingL && npw >= 1 && npw <= kRingNpw && pol >= EMU_POL_TE &&
         pol <= EMU_POL_LCIRC && h->period > 0 && h->period_y > 0 && h->wl_nm > 0;
}

// warp copies of n16 16-byte words; host memory is read with loads that
// bypass the caches (the slot held another request before)
__device__ __forceinline__ void copy_in(int4 *dst, const int4 *src, size_t n16, int lane) {
  for (size_t i = lane; i < n16; i += 32) dst[i] = __ldcv(src + i);
}
__device__ __forceinline__ void copy_out(int4 *dst, const int4 *src, size_t n16, int lane) {
  for (size_t i = lane; i < n16; i += 32) dst[i] = src[i];
}

__global__ void __launch_bounds__(kRingThreads, 2) film_ring_kernel(RingArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long gwarp = (long long)blockIdx.x * kRingWarps + warp;
  RingDev *dv = a.dev;

  // ---------------------------------------------------------------- doorbell
  if (gwarp == 0) {
    if (lane == 0) {
      long long last = ld_acquire_sys(&a.ctl->tail);
      st_release_gpu(&dv->tail, (unsigned long long)last);
      unsigned long long t_act = now_ns();
      // hard bound: about 2^36 polls (days at the poll interval); the idle
      // timeout ends the loop long before
      for (long long it = 0; it < (1ll << 36); ++it) {
        if (ld_volatile_i32(&a.ctl->stop)) {
          atomicExch(&dv->stop, 1);
          break;
        }
        const long long t = ld_acquire_sys(&a.ctl->tail);
        const unsigned long long now = now_ns();
        if (t != last) {
          last = t;
          st_release_gpu(&dv->tail, (unsigned long long)t);
          t_act = now;
          continue;
        }
        if (*(volatile unsigned long long *)&dv->head < (unsigned long long)t) t_act = now;
        if (now - t_act > a.idle_ns) {
          *(volatile int32_t *)&a.ctl->exited = 1;
          __threadfence_system();
          const long long t2 = ld_acquire_sys(&a.ctl->tail);
          if (t2 != last) {
            *(volatile int32_t *)&a.ctl->exited = 0;
            __threadfence_system();
            last = t2;
            st_release_gpu(&dv->tail, (unsigned long long)t2);
            t_act = now_ns();
            continue;
          }
          atomicExch(&dv->stop, 2);
          break;
        }
        __nanosleep(a.sleep_ns);
      }
      if (!*(volatile int *)&dv->stop) atomicExch(&dv->stop, 1);
    }
    return;  // the doorbell warp serves no requests
  }

  // ---------------------------------------------------------------- workers
  const SlotSmem S = slot_layout(kRingNpw, kRingL, true);
  unsigned char *base = smem + warp * S.stride;
  unsigned char *stg = a.stage + gwarp * kStageBytes;
  const WarpTeam tm{lane};
  // poll limit: far above the idle time at the poll interval
  const long long max_polls = (long long)(a.idle_ns / (a.sleep_ns > 0 ? a.sleep_ns : 1)) * 64 + (1ll << 20);
  for (;;) {
    long long ticket = -1;
    if (lane == 0) {
      for (long long polls = 0;; ++polls) {
        const unsigned long long h = *(volatile unsigned long long *)&dv->head;
        const unsigned long long t = ld_acquire_gpu(&dv->tail);
        if (h < t) {
          if (atomicCAS(&dv->head, h, h + 1) == h) {
            ticket = (long long)h;
            break;
          }
          continue;
        }
        if (*(volatile int *)&dv->stop) break;
        if (polls > max_polls) {
          atomicExch(&a.ctl->status, EMU_E_TIMEOUT);
          break;
        }
        __nanosleep(a.sleep_ns);
      }
    }
    ticket = __shfl_sync(0xffffffffu, ticket, 0);
    if (ticket < 0) break;
    __threadfence_system();
    unsigned char *slot = a.slots + (size_t)(ticket % a.cap) * kSlotBytes;
    // the header, then only the parts of the inputs this request uses
    copy_in((int4 *)stg, (const int4 *)slot, sizeof(SlotHdr) / 16, lane);
    __syncwarp();
    const SlotHdr *hd = (const SlotHdr *)stg;
    uint32_t *fl = (uint32_t *)(stg + kOffFl);
    const bool ok = request_ok(hd);
    const int npw = ok ? hd->n_pw : 0, L = ok ? hd->n_layers : 0;
    if (ok) {
      const size_t w_ord = (4 * (size_t)npw + 15) / 16;
      copy_in((int4 *)(stg + kOffPx), (const int4 *)(slot + kOffPx), w_ord, lane);
      copy_in((int4 *)(stg + kOffPy), (const int4 *)(slot + kOffPy), w_ord, lane);
      copy_in((int4 *)(stg + kOffN), (const int4 *)(slot + kOffN), (size_t)L, lane);
      copy_in((int4 *)(stg + kOffH), (const int4 *)(slot + kOffH), (8 * (size_t)L + 15) / 16, lane);
      __syncwarp();
      film_point(tm, RingPoint{hd, stg, a.inv_sqrt2, hd->period_y / hd->period}, true, base, S);
    } else if (lane == 0) {
      *fl = EMU_PT_BAD_POINT;
    }
    __syncwarp();
    // R_net, T_net diagonals, then the lists, r and flags (one block)
    copy_out((int4 *)(slot + kOffR), (const int4 *)(stg + kOffR), 2 * (size_t)npw, lane);
    copy_out((int4 *)(slot + kOffT), (const int4 *)(stg + kOffT), 2 * (size_t)npw, lane);
    copy_out((int4 *)(slot + kOffA), (const int4 *)(stg + kOffA), (kOffFl + 8 - kOffA) / 16, lane);
    __threadfence_system();
    __syncwarp();
    if (lane == 0) *(volatile long long *)(slot + kOffDone) = ticket + 1;
  }
}

}  // namespace

// ------------------------------------------------------------------ host
struct EmuFilmRing {
  int device = 0;
  long long cap = 0;
  unsigned char *h_mem = nullptr;  // control block + slots (pinned, mapped)
  unsigned char *d_mem = nullptr;  // device view of h_mem
  RingDev *d_state = nullptr;
  unsigned char *d_stage = nullptr;
  int grid = 0;
  cudaStream_t stream = nullptr;
  bool launched = false;
  long long next = 0;
  std::vector<long long> consumed;  // per slot: last ticket whose result was read
  std::mutex mu;
  double idle_seconds = 1.0;
  unsigned sleep_ns = 500;
  RingCtl *ctl() { return (RingCtl *)h_mem; }
  unsigned char *slot(long long t) { return h_mem + sizeof(RingCtl) + (size_t)(t % cap) * kSlotBytes; }
};

namespace {

int ring_launch(EmuFilmRing *r) {
  RingArgs a;
  a.ctl = (RingCtl *)r->d_mem;
  a.slots = r->d_mem + sizeof(RingCtl);
  a.cap = r->cap;
  a.dev = r->d_state;
  a.stage = r->d_stage;
  a.idle_ns = (unsigned long long)(r->idle_seconds * 1e9);
  a.sleep_ns = r->sleep_ns;
  a.inv_sqrt2 = 1.0 / sqrt(2.0);
  const size_t smem = (size_t)kRingWarps * slot_layout(kRingNpw, kRingL, true).stride;
  film_ring_kernel<<<r->grid, kRingThreads, smem, r->stream>>>(a);
  emu::note_launch();
  r->launched = true;
  return emu::check_launch();
}

// (re)start the loop when it is not running; called with r->mu held
int ring_ensure_running(EmuFilmRing *r) {
  std::atomic_thread_fence(std::memory_order_seq_cst);
  const bool exited = *(volatile int32_t *)&r->ctl()->exited != 0;
  if (r->launched && !exited && cudaStreamQuery(r->stream) == cudaErrorNotReady) return EMU_OK;
  if (r->launched && cudaStreamSynchronize(r->stream) != cudaSuccess) return EMU_E_CUDA;
  *(volatile int32_t *)&r->ctl()->exited = 0;
  *(volatile int32_t *)&r->ctl()->stop = 0;
  if (cudaMemsetAsync(&r->d_state->stop, 0, sizeof(int), r->stream) != cudaSuccess) return EMU_E_CUDA;
  std::atomic_thread_fence(std::memory_order_seq_cst);
  return ring_launch(r);
}

}  // namespace

extern "C" size_t emu_film_ring_slot_bytes(void) { return kSlotBytes; }

extern "C" int emu_film_ring_create(int capacity, double idle_seconds, EmuFilmRing **out) {
  if (!out || capacity < 1 || capacity > (1 << 20) || !(idle_seconds > 0) || idle_seconds > 600)
    return EMU_E_ARG;
  *out = nullptr;
  EmuFilmRing *r = new EmuFilmRing();
  r->cap = capacity;
  r->idle_seconds = idle_seconds;
  if (cudaGetDevice(&r->device) != cudaSuccess) {
    delete r;
    return EMU_E_CUDA;
  }
  const size_t bytes = sizeof(RingCtl) + (size_t)capacity * kSlotBytes;
  int per_sm = 0;
  const size_t smem = (size_t)kRingWarps * slot_layout(kRingNpw, kRingL, true).stride;
  bool ok = cudaFuncSetAttribute(film_ring_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) ==
                cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, film_ring_kernel, kRingThreads, smem) ==
                cudaSuccess &&
            per_sm >= 1;
  // every CTA resident at once: the doorbell and the workers run together
  r->grid = emu::sm_count() * (per_sm > 0 ? per_sm : 1);
  ok = ok && cudaHostAlloc((void **)&r->h_mem, bytes, cudaHostAllocMapped | cudaHostAllocPortable) == cudaSuccess;
  ok = ok && cudaHostGetDevicePointer((void **)&r->d_mem, r->h_mem, 0) == cudaSuccess;
  ok = ok && cudaMalloc((void **)&r->d_state, sizeof(RingDev)) == cudaSuccess;
  ok = ok && cudaMalloc((void **)&r->d_stage, (size_t)r->grid * kRingWarps * kStageBytes) == cudaSuccess;
  ok = ok && cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking) == cudaSuccess;
  if (ok) {
    std::memset(r->h_mem, 0, bytes);
    ok = cudaMemsetAsync(r->d_state, 0, sizeof(RingDev), r->stream) == cudaSuccess &&
         cudaStreamSynchronize(r->stream) == cudaSuccess;
  }
  if (!ok) {
    cudaGetLastError();
    if (r->stream) cudaStreamDestroy(r->stream);
    if (r->d_stage) cudaFree(r->d_stage);
    if (r->d_state) cudaFree(r->d_state);
    if (r->h_mem) cudaFreeHost(r->h_mem);
    delete r;
    return EMU_E_CUDA;
  }
  r->consumed.assign((size_t)capacity, -1);
  // every slot starts free: ticket t may use slot t % cap once t - cap is consumed
  for (long long s = 0; s < capacity; ++s) r->consumed[s] = s - capacity;
  *out = r;
  return EMU_OK;
}

extern "C" int emu_film_ring_stop(EmuFilmRing *r) {
  if (!r) return EMU_E_ARG;
  std::lock_guard<std::mutex> lock(r->mu);
  *(volatile int32_t *)&r->ctl()->stop = 1;
  std::atomic_thread_fence(std::memory_order_seq_cst);
  if (r->launched && cudaStreamSynchronize(r->stream) != cudaSuccess) return EMU_E_CUDA;
  r->launched = false;
  return *(volatile int32_t *)&r->ctl()->status;
}

extern "C" int emu_film_ring_destroy(EmuFilmRing *r) {
  if (!r) return EMU_E_ARG;
  emu_film_ring_stop(r);
  cudaStreamDestroy(r->stream);
  cudaFree(r->d_stage);
  cudaFree(r->d_state);
  cudaFreeHost(r->h_mem);
  delete r;
  return EMU_OK;
}

extern "C" int emu_film_ring_running(EmuFilmRing *r) {
  if (!r) return 0;
  return (r->launched && cudaStreamQuery(r->stream) == cudaErrorNotReady) ? 1 : 0;
}

namespace {
int request_check(const EmuFilmRingRequest *q) {
  if (q->n_layers < 2 || q->n_layers > kRingL || q->n_pw < 1 || q->n_pw > kRingNpw) return EMU_E_SHAPE;
  if (q->pol < EMU_POL_TE || q->pol > EMU_POL_LCIRC || !(q->period > 0) || !(q->period_y > 0) ||
      !(q->wl_nm > 0) || !q->h_px || !q->h_py || !q->h_n || (q->n_layers > 2 && !q->h_heights_nm))
    return EMU_E_ARG;
  return EMU_OK;
}

// Write request q into the next ticket's slot; false when the ring is full.
// Caller holds r->mu and publishes the tail afterwards.
bool slot_write(EmuFilmRing *r, const EmuFilmRingRequest *q, long long *ticket) {
  const long long t = r->next;
  if (r->consumed[(size_t)(t % r->cap)] != t - r->cap) return false;
  unsigned char *s = r->slot(t);
  SlotHdr h{};
  h.n_layers = q->n_layers;
  h.n_pw = q->n_pw;
  h.world_1d = q->world_1d;
  h.pol = q->pol;
  h.period = q->period;
  h.period_y = q->period_y;
  h.wl_nm = q->wl_nm;
  h.kx = q->k_pll[0];
  h.ky = q->k_pll[1];
  std::memcpy(s + kOffHdr, &h, sizeof(h));
  std::memcpy(s + kOffPx, q->h_px, 4 * (size_t)q->n_pw);
  std::memcpy(s + kOffPy, q->h_py, 4 * (size_t)q->n_pw);
  std::memcpy(s + kOffN, q->h_n, 16 * (size_t)q->n_layers);
  if (q->n_layers > 2) std::memcpy(s + kOffH, q->h_heights_nm, 8 * (size_t)(q->n_layers - 2));
  r->next = t + 1;
  *ticket = t;
  return true;
}

void publish_tail(EmuFilmRing *r) {
  std::atomic_thread_fence(std::memory_order_release);
  *(volatile int64_t *)&r->ctl()->tail = r->next;
}
}  // namespace

extern "C" int emu_film_ring_submit(EmuFilmRing *r, const EmuFilmRingRequest *q, long long *ticket) {
  if (!r || !q || !ticket) return EMU_E_ARG;
  const int st = request_check(q);
  if (st != EMU_OK) return st;
  std::lock_guard<std::mutex> lock(r->mu);
  if (!slot_write(r, q, ticket)) return EMU_E_WORKSPACE;  // ring full
  publish_tail(r);
  return ring_ensure_running(r);
}

extern "C" int emu_film_ring_submit_many(EmuFilmRing *r, const EmuFilmRingRequest *q, int n, long long *tickets,
                                         int *n_submitted) {
  if (!r || n < 0 || (n > 0 && (!q || !tickets)) || !n_submitted) return EMU_E_ARG;
  *n_submitted = 0;
  if (n == 0) return EMU_OK;
  std::lock_guard<std::mutex> lock(r->mu);
  // each request is checked as it is written: the ones before a bad
  // request are submitted, and its status is returned
  int k = 0, st = EMU_OK;
  for (; k < n; ++k) {
    st = request_check(q + k);
    if (st != EMU_OK || !slot_write(r, q + k, tickets + k)) break;
  }
  *n_submitted = k;
  if (k == 0) return st != EMU_OK ? st : EMU_E_WORKSPACE;  // bad first request, or the ring is full
  publish_tail(r);
  const int run = ring_ensure_running(r);
  return run != EMU_OK ? run : st;
}

namespace {
// 1 when the ticket's result is in its slot, 0 when not yet (restarting the
// loop if a request raced its idle end), negative on a bad ticket or error.
// Caller holds r->mu.
int ring_ready(EmuFilmRing *r, long long ticket) {
  if (ticket < 0 || ticket >= r->next || ticket < r->next - r->cap) return -EMU_E_ARG;
  if (r->consumed[(size_t)(ticket % r->cap)] >= ticket) return -EMU_E_ARG;  // already read
  const long long done = *(volatile long long *)(r->slot(ticket) + kOffDone);
  if (done != ticket + 1) {
    if (*(volatile int32_t *)&r->ctl()->exited && cudaStreamQuery(r->stream) != cudaErrorNotReady) {
      const int st = ring_ensure_running(r);  // a request raced the idle end
      if (st != EMU_OK) return -st;
    }
    return 0;
  }
  return 1;
}
}  // namespace

extern "C" int emu_film_ring_ready(EmuFilmRing *r, long long ticket) {
  if (!r) return -EMU_E_ARG;
  std::lock_guard<std::mutex> lock(r->mu);
  return ring_ready(r, ticket);
}

extern "C" int emu_film_ring_poll(EmuFilmRing *r, long long ticket, EmuFilmRingResult *out) {
  if (!r || ticket < 0) return -EMU_E_ARG;
  std::lock_guard<std::mutex> lock(r->mu);
  const int ready = ring_ready(r, ticket);
  if (ready != 1) return ready;
  unsigned char *s = r->slot(ticket);
  std::atomic_thread_fence(std::memory_order_acquire);
  const SlotHdr *h = (const SlotHdr *)(s + kOffHdr);
  if (out) {
    const int P = 2 * h->n_pw, L = h->n_layers;
    if (out->h_R_net) std::memcpy(out->h_R_net, s + kOffR, 16 * (size_t)P);
    if (out->h_T_net) std::memcpy(out->h_T_net, s + kOffT, 16 * (size_t)P);
    if (out->h_a_list) std::memcpy(out->h_a_list, s + kOffA, 8 * (size_t)(L - 1));
    if (out->h_t_list) std::memcpy(out->h_t_list, s + kOffTl, 8 * (size_t)(L - 1));
    if (out->h_r_list) std::memcpy(out->h_r_list, s + kOffRl, 8);
    if (out->h_flags) std::memcpy(out->h_flags, s + kOffFl, 4);
  }
  r->consumed[(size_t)(ticket % r->cap)] = ticket;
  return 1;
}

extern "C" int emu_film_ring_poll_many(EmuFilmRing *r, const long long *tickets, int n,
                                       const EmuFilmRingResult *outs, int32_t *done) {
  if (!r || n < 0 || (n > 0 && (!tickets || !outs || !done))) return -EMU_E_ARG;
  int count = 0;
  for (int i = 0; i < n; ++i) {
    const int st = emu_film_ring_poll(r, tickets[i], const_cast<EmuFilmRingResult *>(outs + i));
    if (st < 0) return st;
    done[i] = st == 1 ? 1 : 0;
    count += done[i];
  }
  return count;
}

extern "C" int emu_film_ring_wait(EmuFilmRing *r, long long ticket, double timeout_s, EmuFilmRingResult *out) {
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    const int st = emu_film_ring_poll(r, ticket, out);
    if (st != 0) return st;
    if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > timeout_s)
      return -EMU_E_TIMEOUT;
    std::this_thread::yield();
  }
}
