"""Continuous-batching server for GSM solves on one GPU.

Requests (one spectral point of a stack each) arrive at any time; a
scheduler thread groups the waiting ones by shape signature, admits as many
as fit the HBM budget into one device batch, and launches it on a free
stream while earlier batches are still running.  Each batch is one fused
launch of the film kernel (``emu_film_stack_batch``) between an async
host-to-device copy of its inputs and a device-to-host copy of its results;
a request's latency runs from ``submit`` to the moment the scheduler sees
its batch's completion event.  Results do not depend on the batch a point
lands in (the film kernel treats every point independently, in a fixed
order of operations), which ``tests/test_gpu_serving.py`` checks.
"""
from __future__ import annotations

import collections
import concurrent.futures as cf
import queue
import threading
import time

import numpy as np
import torch

from .films import FilmStackSolver


class FilmRequest(object):
    """One spectral point of an all-film stack (bottom-to-top indices n)."""

    __slots__ = ('n', 'heights', 'wl_nm', 'k_pll', 'period', 'period_y', 'max_order', 'pol',
                 'world_1d', 'signature', 't_submit', 'future')

    def __init__(self, n, heights, wl_nm, k_pll, period, max_order, pol='TE', period_y=None,
                 world_1d=False):
        self.n = np.asarray(n, np.complex128)
        self.heights = np.asarray(heights, np.float64)
        if self.heights.shape != (len(self.n) - 2,):
            raise ValueError('need one height per finite layer')
        self.wl_nm = float(wl_nm)
        self.k_pll = np.asarray(k_pll, np.float64).reshape(2)
        self.period = float(period)
        self.period_y = float(period if period_y is None else period_y)
        self.max_order = int(max_order)
        self.pol = pol
        self.world_1d = bool(world_1d)
        self.signature = ('film', len(self.n), self.max_order, self.period, self.period_y,
                          self.world_1d, pol)

    def bytes_on_device(self):
        L = len(self.n)
        npw_est = (2 * self.max_order + 1) ** 2
        P = 2 * npw_est
        return 8 + 16 + 16 * L + 8 * (L - 2) + 2 * 16 * P + 2 * 8 * (L - 1) + 12 + L * 160


class _Batch(object):
    def __init__(self, reqs, slot, event, outs, nbytes):
        self.reqs, self.slot, self.event, self.outs, self.nbytes = reqs, slot, event, outs, nbytes


class GsmServer(object):
    """Continuous batching of GSM solve requests on one GPU.

    hbm_budget_bytes bounds the device memory of batches in flight;
    n_streams batches may run at once; max_batch caps one launch.
    """

    def __init__(self, device=None, hbm_budget_bytes=150 << 30, max_batch=32768, n_streams=2,
                 poll_s=2e-4):
        self.device = (torch.device('cuda', torch.cuda.current_device()) if device is None
                       else torch.device(device))
        self.budget = int(hbm_budget_bytes)
        self.max_batch = int(max_batch)
        self.poll_s = poll_s
        self.q = queue.Queue()
        self.pending = collections.OrderedDict()
        self.slots = [dict(stream=torch.cuda.Stream(device=self.device), solvers={}, busy=False)
                      for _ in range(n_streams)]
        self.inflight = []
        self.inflight_bytes = 0
        self.latencies = []
        self.n_batches = 0
        self.batch_sizes = []
        self._stop = threading.Event()
        self._thread = None
        self.t_first = None
        self.t_last = None

    # ---------------------------------------------------------------- API
    def submit(self, req):
        req.future = cf.Future()
        req.t_submit = time.perf_counter()
        if self.t_first is None:
            self.t_first = req.t_submit
        self.q.put(req)
        return req.future

    def start(self):
        self._thread = threading.Thread(target=self._loop, name='gsm-server', daemon=True)
        self._thread.start()
        return self

    def stop(self):
        self._stop.set()
        if self._thread is not None:
            self._thread.join()

    def __enter__(self):
        return self.start()

    def __exit__(self, *a):
        self.stop()

    def stats(self):
        lat = np.array(self.latencies) * 1e3
        n = len(lat)
        span = (self.t_last - self.t_first) if n and self.t_last else float('nan')
        return {
            'requests': n,
            'batches': self.n_batches,
            'mean_batch': float(np.mean(self.batch_sizes)) if self.batch_sizes else 0.0,
            'throughput_per_s': n / span if n and span > 0 else float('nan'),
            'p50_ms': float(np.percentile(lat, 50)) if n else float('nan'),
            'p99_ms': float(np.percentile(lat, 99)) if n else float('nan'),
        }

    # ---------------------------------------------------------------- loop
    def _loop(self):
        torch.cuda.set_device(self.device)
        while True:
            got = False
            while True:
                try:
                    r = self.q.get_nowait()
                except queue.Empty:
                    break
                self.pending.setdefault(r.signature, collections.deque()).append(r)
                got = True
            done_any = self._retire()
            launched = self._launch()
            if self._stop.is_set() and not self.pending and not self.inflight and self.q.empty():
                break
            if not (got or done_any or launched):
                if self.inflight:
                    time.sleep(self.poll_s)
                else:
                    try:
                        r = self.q.get(timeout=0.01)
                        self.pending.setdefault(r.signature, collections.deque()).append(r)
                    except queue.Empty:
                        pass

    def _retire(self):
        done_any = False
        keep = []
        for b in self.inflight:
            if b.event.query():
                t = time.perf_counter()
                host = {k: v.numpy() for k, v in b.outs.items()}
                for i, r in enumerate(b.reqs):
                    res = {k: v[i].copy() for k, v in host.items()}
                    self.latencies.append(t - r.t_submit)
                    r.future.set_result(res)
                self.t_last = t
                self.inflight_bytes -= b.nbytes
                b.slot['busy'] = False
                done_any = True
            else:
                keep.append(b)
        self.inflight = keep
        return done_any

    def _launch(self):
        launched = False
        for slot in self.slots:
            if slot['busy'] or not self.pending:
                continue
            sig = next(iter(self.pending))
            dq = self.pending[sig]
            reqs, nbytes = [], 0
            while dq and len(reqs) < self.max_batch:
                nb = dq[0].bytes_on_device()
                if self.inflight_bytes + nbytes + nb > self.budget and reqs:
                    break
                if self.inflight_bytes + nbytes + nb > self.budget and self.inflight:
                    break
                reqs.append(dq.popleft())
                nbytes += nb
            if not dq:
                del self.pending[sig]
            else:
                self.pending.move_to_end(sig)
            if not reqs:
                continue
            self._run_batch(slot, sig, reqs, nbytes)
            launched = True
        return launched

    def _run_batch(self, slot, sig, reqs, nbytes):
        _, L, mo, per, per_y, w1d, pol = sig
        B = len(reqs)
        solver = slot['solvers'].get(sig)
        if solver is None:
            solver = FilmStackSolver(L, mo, per, per_y, w1d, device=self.device)
            slot['solvers'][sig] = solver
        wl = torch.empty(B, dtype=torch.float64).pin_memory()
        kp = torch.empty((B, 2), dtype=torch.float64).pin_memory()
        n = torch.empty((B, L), dtype=torch.complex128).pin_memory()
        h = torch.empty((B, max(L - 2, 0)), dtype=torch.float64).pin_memory()
        wl.numpy()[:] = [r.wl_nm for r in reqs]
        kp.numpy()[:] = np.stack([r.k_pll for r in reqs])
        n.numpy()[:] = np.stack([r.n for r in reqs])
        if L > 2:
            h.numpy()[:] = np.stack([r.heights for r in reqs])
        s = slot['stream']
        with torch.cuda.stream(s):
            dwl = wl.to(self.device, non_blocking=True)
            dkp = kp.to(self.device, non_blocking=True)
            dn = n.to(self.device, non_blocking=True)
            dh = h.to(self.device, non_blocking=True) if L > 2 else None
            o = solver.solve(dwl, dkp, dn, dh, pol=pol, stream=s)
            outs = {}
            for k in ('R_net', 'T_net', 'a_list', 't_list', 'r_list', 'flags'):
                t = torch.empty(o[k].shape, dtype=o[k].dtype).pin_memory()
                t.copy_(o[k], non_blocking=True)
                outs[k] = t
            ev = torch.cuda.Event()
            ev.record(s)
        # keep the device inputs alive until the batch retires
        outs_keep = _Batch(reqs, slot, ev, outs, nbytes)
        outs_keep.keep = (dwl, dkp, dn, dh)
        slot['busy'] = True
        self.inflight.append(outs_keep)
        self.inflight_bytes += nbytes
        self.n_batches += 1
        self.batch_sizes.append(B)
