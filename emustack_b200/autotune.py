"""Launch-configuration autotuner.

Kernels of this package expose launch choices that never change results,
only speed: the film kernel's CTA shape (``EmuFilmStackBatch.variant``), the
uneven-batch kernel's warps per CTA, the tensor-core overlap path's element
chunk and K splits.  The best choice depends on the shape (orders, layers,
batch size, mesh size) and on the GPU, so it is measured, not guessed: the
first call for a shape times every candidate with CUDA events on the
caller's stream (after a warm-up launch each) and keeps the fastest; later
calls reuse it.

Choices are cached per (GPU name, kernel family, shape key) in memory and,
if ``EMUSTACK_AUTOTUNE_CACHE`` names a file (or a path is given), in that
JSON file, so a serving process starts tuned.  ``EMUSTACK_AUTOTUNE=0``
disables tuning (every caller then uses its default).
"""
from __future__ import annotations

import json
import os
import warnings
import threading

import torch


class Autotuner(object):
    """time_fn(run, choice, stream) -> milliseconds per launch; the default
    times ``reps`` launches with CUDA events after ``warmup`` launches."""

    def __init__(self, path=None, warmup=1, reps=3, time_fn=None, tie=0.02):
        self.path = path if path is not None else _ENV_PATH
        if self.path:
            self.path = os.path.abspath(self.path)
        self.tie = float(tie)
        self.time_fn = time_fn or self._cuda_time
        self.enabled = os.environ.get('EMUSTACK_AUTOTUNE', '1') != '0'
        self.warmup, self.reps = warmup, reps
        self.cache = {}
        self.log = []
        self._lock = threading.Lock()
        if self.path and os.path.exists(self.path):
            try:
                with open(self.path) as f:
                    self.cache = json.load(f)
            except (OSError, ValueError):
                self.cache = {}

    @staticmethod
    def _key(family, shape):
        dev = (torch.cuda.get_device_name(torch.cuda.current_device())
               if torch.cuda.is_available() else 'cpu')
        return '%s|%s|%s' % (dev, family, json.dumps(shape, sort_keys=True))

    def _cuda_time(self, run, c, stream):
        s = stream if stream is not None else torch.cuda.current_stream()
        with torch.cuda.stream(s):
            for _ in range(self.warmup):
                run(c)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(s)
            for _ in range(self.reps):
                run(c)
            b.record(s)
            b.synchronize()
        return a.elapsed_time(b) / self.reps

    def choose(self, family, shape, candidates, run, default, stream=None):
        """Return the fastest of ``candidates`` for this shape.

        run(c) launches the work once with choice c on the current stream
        (it must leave results identical for every c).  Without tuning the
        default is returned.
        """
        if not self.enabled or len(candidates) < 2:
            return default
        key = self._key(family, shape)
        with self._lock:
            hit = self.cache.get(key)
        if hit is not None:
            return _as_choice(hit['choice'])
        times, errors = {}, {}
        for c in candidates:
            try:
                times[json.dumps(c)] = self.time_fn(run, c, stream)
            except Exception as e:  # a choice this shape cannot launch with
                errors[json.dumps(c)] = e
        if not times:
            raise next(iter(errors.values()))
        # the first candidate (in the caller's order) within `tie` of the
        # fastest: near-equal timings do not flip the choice from run to run
        fastest = min(times.values())
        best = next(k for k in times if times[k] <= fastest * (1.0 + self.tie))
        entry = {'choice': json.loads(best), 'ms': times}
        with self._lock:
            self.cache[key] = entry
            self.log.append((key, entry))
            if self.path:
                tmp = self.path + '.tmp'
                try:
                    with open(tmp, 'w') as f:
                        json.dump(self.cache, f, indent=1, sort_keys=True)
                    os.replace(tmp, self.path)
                except OSError as e:   # the choice stands; only its record is lost
                    warnings.warn('autotune cache %s not written: %s' % (self.path, e))
        return _as_choice(entry['choice'])


def _as_choice(c):
    return tuple(c) if isinstance(c, list) else c


_default = None
# the cache file named by the environment, resolved against the working
# directory at import, so that later directory changes keep the same file
_ENV_PATH = os.environ.get('EMUSTACK_AUTOTUNE_CACHE')
if _ENV_PATH:
    _ENV_PATH = os.path.abspath(_ENV_PATH)


def default_tuner():
    global _default
    if _default is None:
        _default = Autotuner()
    return _default


def size_bucket(n):
    """Power-of-two bucket of a batch or mesh size (tuned choices are shared
    by sizes within a factor of two)."""
    n = max(int(n), 1)
    return 1 << (n - 1).bit_length()
