// Library-wide C-ABI functions: version, status strings, launch counter and
// the plane-wave order set (host integer/IEEE bookkeeping, no kernel).
#include <atomic>
#include <mutex>

#include "emu_internal.h"

namespace emu {

static std::atomic<long long> g_launches{0};
static std::atomic<int> g_dense_mode{0};

void note_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int dense_mode() { return g_dense_mode.load(std::memory_order_relaxed); }

int sm_count() {
  static int cache[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (cache[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
      n = 148;
    cache[dev] = n;
  }
  return cache[dev];
}

}  // namespace emu

extern "C" {

int emu_version(void) { return 100; }

long long emu_launch_count(void) { return emu::g_launches.load(); }

int emu_set_dense_mode(int mode) {
  if (mode < 0 || mode > 2) return -1;
  return emu::g_dense_mode.exchange(mode);
}

const char *emu_status_string(int s) {
  switch (s) {
    case EMU_OK: return "EMU_OK";
    case EMU_E_ARG: return "EMU_E_ARG: invalid argument";
    case EMU_E_SHAPE: return "EMU_E_SHAPE: unsupported or inconsistent dimensions";
    case EMU_E_SINGULAR: return "EMU_E_SINGULAR: singular matrix";
    case EMU_E_NONFINITE: return "EMU_E_NONFINITE: non-finite result";
    case EMU_E_WORKSPACE: return "EMU_E_WORKSPACE: workspace too small";
    case EMU_E_TIMEOUT: return "EMU_E_TIMEOUT: bounded device wait gave up";
    case EMU_E_CUDA: return "EMU_E_CUDA: CUDA runtime error";
    case EMU_E_UNSUPPORTED: return "EMU_E_UNSUPPORTED: unsupported request";
    default: return "unknown status";
  }
}

// The disc test is evaluated exactly as numpy evaluates
//   (pxs/dx)**2 + (pys/dy)**2 <= (max_order/max(dx, dy))**2
// (backend/mode_calcs.py:72-73): one rounding per operation, no fused
// multiply-add (this file is compiled with -ffp-contract=off for the host).
int emu_grating_orders(int max_order, double period, double period_y, int world_1d,
                       int32_t *h_px, int32_t *h_py, int capacity, int *h_count) {
  if (max_order < 0 || !(period > 0) || !(period_y > 0) || h_count == nullptr) return EMU_E_ARG;
  int n = 0;
  if (world_1d) {
    for (int px = -max_order; px <= max_order; ++px) {
      if (h_px && n < capacity) {
        h_px[n] = px;
        if (h_py) h_py[n] = 0;
      }
      ++n;
    }
  } else {
    const double dx = period, dy = period_y;
    const double mxd = dx > dy ? dx : dy;
    volatile double rq = (double)max_order / mxd;
    const double r2 = rq * rq;
    for (int px = -max_order; px <= max_order; ++px) {
      for (int py = -max_order; py <= max_order; ++py) {
        volatile double a = (double)px / dx;
        volatile double b = (double)py / dy;
        volatile double a2 = a * a;
        volatile double b2 = b * b;
        volatile double s = a2 + b2;
        if (s <= r2) {
          if (h_px && n < capacity) {
            h_px[n] = px;
            if (h_py) h_py[n] = py;
          }
          ++n;
        }
      }
    }
  }
  *h_count = n;
  if ((h_px || h_py) && n > capacity) return EMU_E_SHAPE;
  return EMU_OK;
}

}  // extern "C"
