"""Measured FP64 FMA peak of the current GPU (DFMA probe kernel)."""
from __future__ import annotations

import ctypes as C

from ._lib import check, lib, ptr, stream_ptr, EXTRA_SIGNATURES, vp

EXTRA_SIGNATURES.append(('emu_probe_fp64', C.c_int, [C.c_int, C.c_int, C.c_int, vp, vp]))

_cache = {}


def fp64_peak_tflops(iters=4096):
    """Best of 5 timed runs of 64 FMA chains per thread on every SM."""
    import torch
    dev = torch.cuda.current_device()
    if dev in _cache:
        return _cache[dev]
    L = lib()
    f = L.emu_probe_fp64
    f.restype, f.argtypes = C.c_int, [C.c_int, C.c_int, C.c_int, vp, vp]
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    blocks, threads = sms * 8, 256
    out = torch.empty(blocks, dtype=torch.float64, device='cuda')
    best = 0.0
    for _ in range(6):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        check(f(blocks, threads, iters, ptr(out), stream_ptr()), 'emu_probe_fp64')
        e.record()
        torch.cuda.synchronize()
        ms = s.elapsed_time(e)
        best = max(best, 2.0 * 64 * iters * threads * blocks / (ms / 1e3) / 1e12)
    _cache[dev] = best
    return best
