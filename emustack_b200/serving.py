"""Continuous-batching server for GSM solves on one GPU.

Requests -- one spectral point each, of an all-film stack of any shape
(``FilmRequest``) or of a stack with nanostructured array layers
(``ArrayRequest``, emustack_b200.array_serving) -- arrive at any time; a
scheduler thread admits waiting requests into a device batch as long as the
batch fits the HBM budget left by the batches still in flight, and launches
it on a free stream while earlier batches are still running.  Array layers'
interfaces with the air reference are cached on the device (``SMatrixCache``)
and reused by every later request that names the same layer.

Film requests have two batching modes:

* ``'mixed'`` (default): a batch takes requests in arrival order whatever
  their shape (layer count, order set, periods, polarisation) and runs as one
  launch of the uneven-batch film kernel (``emu_film_var_batch``, one warp
  per point);
* ``'grouped'``: requests are grouped by shape signature and each batch is
  one launch of the uniform film kernel (``emu_film_stack_batch``).

Array requests whose matrices are small (D = max(P, M) <= uneven_max_dim)
share one uneven batch whatever their shapes: film modes and missing
interfaces per order set, then every cascade in ONE launch of the uneven
dense kernel (``ArrayBatcher.launch_uneven``, one CTA per stack).  Larger
ones are grouped by shape signature (order set, polarisation, layer kinds
and Bloch-mode counts) and each group's cascade spreads over the GPU
(``ArrayBatcher.launch``).

Each batch is an async host-to-device copy of its packed inputs, one kernel,
and an async device-to-host copy of its packed outputs on the slot's
stream.  A request's latency runs from its arrival (``t_arrival`` if the
caller scheduled one, else ``submit``) to the moment the scheduler sees its
batch's completion event.  Results do not depend on the batch a point lands
in: the kernels treat every point independently, with one fixed order of
operations per point.
"""
from __future__ import annotations

import collections
import ctypes as C
import itertools
import threading
import time

import numpy as np
import torch

from .array_serving import (ArrayBatcher, ArrayLayer, ArrayRequest, SMatrixCache,  # noqa: F401
                            dense_workspace_bytes)
from . import _lib
from ._lib import check
from .films import FilmPoint, FilmStackSolver, FilmVarSolver, grating_orders

_NPW = {}


def _npw(max_order, period, period_y, world_1d):
    key = (max_order, period, period_y, world_1d)
    n = _NPW.get(key)
    if n is None:
        n = len(grating_orders(max_order, period, period_y, world_1d)[0])
        _NPW[key] = n
    return n


class FilmRequest(FilmPoint):
    """One spectral point of an all-film stack (bottom-to-top indices n)."""

    __slots__ = ('signature', 't_submit', 't_arrival', 'future', 'npw')

    def __init__(self, n, heights, wl_nm, k_pll, period, max_order, pol='TE', period_y=None,
                 world_1d=False, incoming=None, t_arrival=None):
        super().__init__(n, heights, wl_nm, k_pll, period, max_order, pol=pol, period_y=period_y,
                         world_1d=world_1d, incoming=incoming)
        self.npw = _npw(self.max_order, self.period, self.period_y, self.world_1d)
        self.signature = ('film', len(self.n), self.max_order, self.period, self.period_y,
                          self.world_1d, pol if incoming is None else None)
        self.t_arrival = t_arrival

    def bytes_on_device(self):
        """Inputs, outputs and workspace of this point on the device."""
        L, P = len(self.n), 2 * self.npw
        slots = self.npw if self.incoming is not None else 1
        return (120 + 16 * L + 8 * (L - 2) + (16 * P if self.incoming is not None else 0)
                + 2 * 16 * P + 2 * 8 * (L - 1) + 4 * (L + 1) + 16 + slots * L * 160)


class FilmResult(object):
    """Outputs of one request: dict-like view into its batch's host arrays
    (keys R_net, T_net, a_list, t_list, r_list, flags, specular)."""

    __slots__ = ('_h', '_ro', '_P', '_lo', '_L', '_i')

    def __init__(self, host, ro, P, lo, L, i):
        self._h, self._ro, self._P, self._lo, self._L, self._i = host, ro, P, lo, L, i

    def __getitem__(self, k):
        h = self._h
        if k in ('R_net', 'T_net'):
            return h[k][self._ro:self._ro + self._P]
        if k in ('a_list', 't_list'):
            return h[k][self._lo:self._lo + self._L - 1]
        if k == 'r_list':
            return h['r_list'][self._i]
        if k in ('flags', 'specular'):
            return int(h[k][self._i])
        raise KeyError(k)

    def keys(self):
        return ('R_net', 'T_net', 'a_list', 't_list', 'r_list', 'flags', 'specular')


class RequestFuture(object):
    """Completion handle of one request (the subset of concurrent.futures.
    Future the server needs, without a lock per request: completions are
    published per batch under the server's one condition variable)."""

    __slots__ = ('_value', '_exc', '_done', '_cv')

    def __init__(self, cv):
        self._cv = cv
        self._done = False
        self._value = self._exc = None

    def done(self):
        return self._done

    def result(self, timeout=None):
        if not self._done:
            end = None if timeout is None else time.monotonic() + timeout
            with self._cv:
                while not self._done:
                    left = None if end is None else end - time.monotonic()
                    if left is not None and left <= 0:
                        raise TimeoutError('request not finished')
                    self._cv.wait(left)
        if self._exc is not None:
            raise self._exc
        return self._value


class _Batch(object):
    __slots__ = ('reqs', 'slot', 'event', 'nbytes', 'finish', 'keep')

    def __init__(self, reqs, slot, event, nbytes, finish, keep):
        self.reqs, self.slot, self.event = reqs, slot, event
        self.nbytes, self.finish, self.keep = nbytes, finish, keep


class GsmServer(object):
    """Continuous batching of GSM solve requests on one GPU.

    hbm_budget_bytes bounds the device memory of the server: the layer
    interface cache (smatrix_cache_bytes of it; default an eighth, at most
    16 GiB) plus the batches in flight; array requests with D = max(P, M) <=
    uneven_max_dim share one-launch uneven batches whose workspace is at most
    uneven_ws_bytes;
    n_streams batches may run at once; max_batch caps one launch;
    batching of film requests is 'mixed' (any shapes in one launch) or
    'grouped'.
    """

    def __init__(self, device=None, hbm_budget_bytes=150 << 30, max_batch=32768, n_streams=2,
                 poll_s=2e-4, batching='mixed', smatrix_cache_bytes=None, uneven_max_dim=256,
                 uneven_ws_bytes=8 << 30):
        if batching not in ('mixed', 'grouped'):
            raise ValueError("batching must be 'mixed' or 'grouped'")
        self.device = (torch.device('cuda', torch.cuda.current_device()) if device is None
                       else torch.device(device))
        self.batching = batching
        if smatrix_cache_bytes is None:
            smatrix_cache_bytes = min(16 << 30, int(hbm_budget_bytes) // 8)
        if smatrix_cache_bytes >= hbm_budget_bytes:
            raise ValueError('the layer interface cache must leave room for batches in the budget')
        self.cache = SMatrixCache(smatrix_cache_bytes)
        self._arrays = None
        self._launcher = None
        self.max_array_slots = max(1, n_streams - 1)
        self.uneven_max_dim = int(uneven_max_dim)
        self.uneven_ws_bytes = int(uneven_ws_bytes)
        self.budget = int(hbm_budget_bytes) - int(smatrix_cache_bytes)
        self.max_batch = int(max_batch)
        self.poll_s = poll_s
        self.q = collections.deque()      # submit -> scheduler (append / popleft are atomic)
        self._wake = threading.Event()
        self._idle = False
        self._cv = threading.Condition()
        self.pending = collections.OrderedDict()
        self.slots = [dict(stream=torch.cuda.Stream(device=self.device), solvers={}, busy=False,
                           var=None) for _ in range(n_streams)]
        self.inflight = []
        self.inflight_bytes = 0
        self.latencies = []
        self.array_latencies = []         # the array requests' share of latencies
        self.n_batches = 0
        self.batch_sizes = []
        self._stop = threading.Event()
        self._thread = None
        self.t_first = None
        self.t_last = None
        self.error = None
        # host seconds spent packing, launching and finishing batches, and
        # device seconds from the H2D copy to the end of the D2H copy
        self.prof = dict(plan_s=0.0, launch_s=0.0, finish_s=0.0, device_s=0.0)

    # ---------------------------------------------------------------- API
    def submit(self, req):
        req.future = RequestFuture(self._cv)
        req.t_submit = time.perf_counter()
        t0 = req.t_arrival if req.t_arrival is not None else req.t_submit
        if self.t_first is None or t0 < self.t_first:
            self.t_first = t0
        self.q.append(req)
        if self._idle:
            self._wake.set()
        return req.future

    def start(self):
        self._thread = threading.Thread(target=self._loop, name='gsm-server', daemon=True)
        self._thread.start()
        return self

    def stop(self):
        self._stop.set()
        self._wake.set()
        if self._thread is not None:
            self._thread.join()
        if self._launcher is not None:
            self._launcher.shutdown(wait=True)
            self._launcher = None

    def __enter__(self):
        return self.start()

    def __exit__(self, *a):
        self.stop()

    def stats(self):
        lat = np.array(self.latencies) * 1e3
        n = len(lat)
        span = (self.t_last - self.t_first) if n and self.t_last else float('nan')
        alat = np.array(self.array_latencies) * 1e3
        pct = lambda a, q: float(np.percentile(a, q)) if len(a) else float('nan')
        return {
            'requests': n,
            'batches': self.n_batches,
            'mean_batch': float(np.mean(self.batch_sizes)) if self.batch_sizes else 0.0,
            'throughput_per_s': n / span if n and span > 0 else float('nan'),
            'p50_ms': pct(lat, 50),
            'p99_ms': pct(lat, 99),
            'array_requests': len(alat),
            'array_p50_ms': pct(alat, 50),
            'array_p99_ms': pct(alat, 99),
            'smatrix_cache': self.cache.stats(),
        }

    # ---------------------------------------------------------------- loop
    def _key(self, r):
        if isinstance(r, ArrayRequest):
            return 'array-uneven' if r.max_dim() <= self.uneven_max_dim else r.signature
        return 'all' if self.batching == 'mixed' else r.signature

    def _take(self, block):
        if block and not self.q:
            self._idle = True
            if not self.q:
                self._wake.wait(0.01)
            self._idle = False
            self._wake.clear()
        got = False
        q, pend = self.q, self.pending
        while q:
            r = q.popleft()
            k = self._key(r)
            d = pend.get(k)
            if d is None:
                d = pend[k] = collections.deque()
            d.append(r)
            got = True
        return got

    def _loop(self):
        torch.cuda.set_device(self.device)
        try:
            while True:
                got = self._take(block=False)
                done_any = self._retire()
                launched = self._launch()
                if self._stop.is_set() and not self.pending and not self.inflight and not self.q:
                    break
                if not (got or done_any or launched):
                    if self.inflight:
                        time.sleep(self.poll_s)
                    else:
                        self._take(block=True)
        except Exception as e:  # fail every waiting request instead of hanging them
            self.error = e
            waiting = [r for b in self.inflight for r in b.reqs]
            waiting += [r for dq in self.pending.values() for r in dq]
            while self.q:
                waiting.append(self.q.popleft())
            self._publish([r for r in waiting if not r.future.done()], exc=e)

    def _publish(self, reqs, values=None, exc=None):
        """Complete a batch of requests and wake their waiters once."""
        with self._cv:
            for i, r in enumerate(reqs):
                f = r.future
                if exc is not None:
                    f._exc = exc
                else:
                    f._value = values[i]
                f._done = True
            self._cv.notify_all()

    def _retire(self):
        done_any = False
        keep = []
        for b in self.inflight:
            if b.event is None:
                # a shape group whose launches a worker thread is still issuing
                if not b.keep.done():
                    keep.append(b)
                    continue
                try:
                    b.event, fin = b.keep.result()
                except Exception as e:  # the launch failed: fail its requests only
                    self._publish(b.reqs, exc=e)
                    self.inflight_bytes -= b.nbytes
                    b.slot['busy'] = False
                    done_any = True
                    continue
                b.finish = self._array_finish(fin)
            if b.event.query():
                t = time.perf_counter()
                b.finish(b, t)
                self.t_last = t
                self.inflight_bytes -= b.nbytes
                b.slot['busy'] = False
                done_any = True
            else:
                keep.append(b)
        self.inflight = keep
        return done_any

    def _is_array_key(self, key):
        return key == 'array-uneven' or (isinstance(key, tuple) and key[0] == 'array')

    def _launch(self):
        launched = False
        for slot in self.slots:
            if slot['busy'] or not self.pending:
                continue
            # array batches may hold at most max_array_slots streams, so film
            # requests always find a stream of their own
            arrays_busy = sum(1 for sl in self.slots if sl['busy'] and sl.get('array'))
            key = None
            for k in self.pending:
                if not self._is_array_key(k) or arrays_busy < self.max_array_slots:
                    key = k
                    break
            if key is None:
                continue
            slot['array'] = self._is_array_key(key)
            dq = self.pending[key]
            reqs, nbytes = [], 0
            while dq and len(reqs) < self.max_batch:
                nb = dq[0].bytes_on_device()
                if self.inflight_bytes + nbytes + nb > self.budget and (reqs or self.inflight):
                    break
                reqs.append(dq.popleft())
                nbytes += nb
            if not dq:
                del self.pending[key]
            else:
                self.pending.move_to_end(key)
            if not reqs:
                continue
            if key == 'array-uneven':
                self._run_arrays(slot, reqs, nbytes, uneven=True)
            elif isinstance(reqs[0], ArrayRequest):
                self._run_arrays(slot, reqs, nbytes)
            elif self.batching == 'mixed':
                self._run_mixed(slot, reqs, nbytes)
            else:
                self._run_grouped(slot, reqs[0].signature, reqs, nbytes)
            launched = True
        return launched

    def _record(self, reqs, t):
        lat = [t - (r.t_arrival if r.t_arrival is not None else r.t_submit) for r in reqs]
        self.latencies.extend(lat)
        if reqs and isinstance(reqs[0], ArrayRequest):
            self.array_latencies.extend(lat)

    def _run_mixed(self, slot, reqs, nbytes):
        if slot['var'] is None:
            slot['var'] = FilmVarSolver(self.device)
        solver = slot['var']
        s = slot['stream']
        t0 = time.perf_counter()
        pl = solver.plan(reqs)
        t1 = time.perf_counter()
        e0 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        out = solver.solve(pl, stream=s)
        host = solver.fetch(out, stream=s)
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(s)
        self.prof['plan_s'] += t1 - t0
        self.prof['launch_s'] += time.perf_counter() - t1
        desc = pl.desc

        def finish(b, t):
            # copy out of the slot's staging buffers before the slot is reused
            t2 = time.perf_counter()
            h = {k: v.copy() for k, v in host.items()}
            ro, lo = desc['rt_off'].tolist(), desc['list_off'].tolist()
            P, L = (2 * desc['n_pw']).tolist(), desc['n_layers'].tolist()
            vals = [FilmResult(h, ro[i], P[i], lo[i], L[i], i) for i in range(len(b.reqs))]
            self._publish(b.reqs, vals)
            self._record(b.reqs, t)
            self.prof['finish_s'] += time.perf_counter() - t2
            self.prof['device_s'] += e0.elapsed_time(b.event) / 1e3

        self._submit(_Batch(reqs, slot, ev, nbytes, finish, None))

    def _run_grouped(self, slot, sig, reqs, nbytes):
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
            o = solver.solve(dwl, dkp, dn, dh, pol=pol, stream=s, want=('specular',))
            outs = {}
            for k in ('R_net', 'T_net', 'a_list', 't_list', 'r_list', 'flags', 'specular'):
                t = torch.empty(o[k].shape, dtype=o[k].dtype).pin_memory()
                t.copy_(o[k], non_blocking=True)
                outs[k] = t
            ev = torch.cuda.Event()
            ev.record(s)

        def finish(b, t):
            host = {k: v.numpy() for k, v in outs.items()}
            vals = [{k: (v[i].copy() if v.ndim > 1 else v[i]) for k, v in host.items()}
                    for i in range(len(b.reqs))]
            self._publish(b.reqs, vals)
            self._record(b.reqs, t)

        self._submit(_Batch(reqs, slot, ev, nbytes, finish, (dwl, dkp, dn, dh)))

    def _run_arrays(self, slot, reqs, nbytes, uneven=False):
        if self._arrays is None:
            self._arrays = ArrayBatcher(self.device, self.cache)
        t1 = time.perf_counter()
        if uneven:
            # the cascade workspace stays within what admission counted for
            # these requests (each counts its own per-solve workspace)
            counted = sum(dense_workspace_bytes(2 * r.npw, [ly.M if isinstance(ly, ArrayLayer) else 2 * r.npw
                                                            for ly in r.layers]) for r in reqs)
            ev, fin = self._arrays.launch_uneven(reqs, slot['stream'], id(slot),
                                                 min(self.uneven_ws_bytes, counted))
            self.prof['launch_s'] += time.perf_counter() - t1
            self._submit(_Batch(reqs, slot, ev, nbytes, self._array_finish(fin), None))
            return
        # a shape group spreads each cascade step over the GPU: thousands of
        # launches for large matrices.  A worker thread per stream issues them
        # (the library releases the interpreter lock while it launches), so
        # the scheduler keeps admitting and retiring other batches meanwhile.
        if self._launcher is None:
            import concurrent.futures as cf
            self._launcher = cf.ThreadPoolExecutor(max_workers=len(self.slots),
                                                   thread_name_prefix='gsm-array-launch')
        dev, stream = self.device, slot['stream']

        def work():
            torch.cuda.set_device(dev)
            return self._arrays.launch(reqs, stream, id(slot))

        fut = self._launcher.submit(work)
        self.prof['launch_s'] += time.perf_counter() - t1
        self._submit(_Batch(reqs, slot, None, nbytes, None, fut))

    def _array_finish(self, fin):
        def finish(b, t):
            t2 = time.perf_counter()
            vals = fin()
            ok = [i for i, v in enumerate(vals) if not isinstance(v, Exception)]
            self._publish([b.reqs[i] for i in ok], [vals[i] for i in ok])
            for i, v in enumerate(vals):
                if isinstance(v, Exception):
                    self._publish([b.reqs[i]], exc=v)
            self._record(b.reqs, t)
            self.prof['finish_s'] += time.perf_counter() - t2

        return finish

    def _submit(self, batch):
        batch.slot['busy'] = True
        self.inflight.append(batch)
        self.inflight_bytes += batch.nbytes
        self.n_batches += 1
        self.batch_sizes.append(len(batch.reqs))


class DeviceFilmServer(object):

    """All-film solves served by a device-resident request loop
    (emu_film_ring_*): a persistent kernel picks requests up from a ring in
    pinned host memory as they are submitted, one warp per request, and
    writes each result back into its slot.  No kernel launch or host
    scheduling thread per request; the loop ends by itself idle_seconds after
    the last request and restarts on the next submit.

    submit(req) takes a FilmRequest (standard polarisation, at most
    EMU_RING_MAX_LAYERS layers and EMU_RING_MAX_PW orders per polarisation)
    and returns a ticket; poll(ticket) returns the result dict once done
    (R_net, T_net diagonals, a_list, t_list, r_list, flags) or None;
    wait(ticket) blocks (outside the interpreter lock) until done.  While the
    loop runs it holds every SM of the device."""

    _REQ = None   # numpy layouts of EmuFilmRingRequest / EmuFilmRingResult
    _RES = None

    def __init__(self, capacity=4096, idle_seconds=1.0):
        self._L = _lib.lib()
        h = C.c_void_p()
        check(self._L.emu_film_ring_create(int(capacity), float(idle_seconds), C.byref(h)),
              'emu_film_ring_create')
        self._h = h
        self._pending = collections.OrderedDict()   # ticket -> (layers, orders), oldest first
        self._early = {}
        self._orders = {}

    def _order_arrays(self, r):
        key = (r.max_order, r.period, r.period_y, r.world_1d)
        o = self._orders.get(key)
        if o is None:
            from .films import grating_orders
            px, py = grating_orders(r.max_order, r.period, r.period_y, r.world_1d)
            o = self._orders[key] = (np.ascontiguousarray(px, np.int32), np.ascontiguousarray(py, np.int32))
        return o

    def submit(self, r):
        if r.incoming is not None:
            raise ValueError('the device request loop takes standard polarisations only')
        px, py = self._order_arrays(r)
        n = np.ascontiguousarray(r.n, np.complex128)
        h = np.ascontiguousarray(r.heights, np.float64)
        q = _lib.EmuFilmRingRequest()
        q.n_layers, q.n_pw, q.world_1d, q.pol = len(n), len(px), int(bool(r.world_1d)), _lib.POL[r.pol]
        q.period, q.period_y, q.wl_nm = r.period, r.period_y, r.wl_nm
        q.k_pll[0], q.k_pll[1] = float(r.k_pll[0]), float(r.k_pll[1])
        q.h_px, q.h_py = px.ctypes.data_as(C.c_void_p), py.ctypes.data_as(C.c_void_p)
        q.h_n, q.h_heights_nm = n.ctypes.data_as(C.c_void_p), h.ctypes.data_as(C.c_void_p)
        t = C.c_longlong()
        while True:
            st = self._L.emu_film_ring_submit(self._h, C.byref(q), C.byref(t))
            if st != _lib.EMU_E_WORKSPACE:   # the ring is full until results are read
                break
            self._drain_one()
        check(st, 'emu_film_ring_submit')
        self._pending[t.value] = (len(n), len(px))
        return t.value

    @staticmethod
    def _dtype(cs):
        """numpy layout of a ctypes descriptor (the C struct's offsets)."""
        names, formats, offsets = [], [], []
        for f, t in cs._fields_:
            names.append(f)
            offsets.append(getattr(cs, f).offset)
            if t is C.c_int:
                formats.append(np.int32)
            elif t is C.c_double:
                formats.append(np.float64)
            elif t is C.c_void_p:
                formats.append(np.uintp)
            else:   # c_double * k
                formats.append((np.float64, (t._length_,)))
        return np.dtype({'names': names, 'formats': formats, 'offsets': offsets, 'itemsize': C.sizeof(cs)})

    def submit_many(self, reqs):
        """Submit requests in order with one call into the library per batch
        of free slots; returns their tickets.  When the ring is full the
        oldest results are read first (poll, poll_many, wait and take still
        return them)."""
        reqs = list(reqs)
        if any(r.incoming is not None for r in reqs):
            raise ValueError('the device request loop takes standard polarisations only')
        n = len(reqs)
        if n == 0:
            return []
        if self._REQ is None:
            type(self)._REQ = self._dtype(_lib.EmuFilmRingRequest)
        orders = [self._order_arrays(r) for r in reqs]
        ns = [np.ascontiguousarray(r.n, np.complex128) for r in reqs]
        hs = [np.ascontiguousarray(r.heights, np.float64) for r in reqs]
        a = np.zeros(n, self._REQ)
        a['n_layers'] = [len(x) for x in ns]
        a['n_pw'] = [len(o[0]) for o in orders]
        a['world_1d'] = [int(bool(r.world_1d)) for r in reqs]
        a['pol'] = [_lib.POL[r.pol] for r in reqs]
        a['period'] = [r.period for r in reqs]
        a['period_y'] = [r.period_y for r in reqs]
        a['wl_nm'] = [r.wl_nm for r in reqs]
        a['k_pll'] = [r.k_pll for r in reqs]
        a['h_px'] = [o[0].ctypes.data for o in orders]
        a['h_py'] = [o[1].ctypes.data for o in orders]
        a['h_n'] = [x.ctypes.data for x in ns]
        a['h_heights_nm'] = [x.ctypes.data for x in hs]
        tickets = np.empty(n, np.int64)
        done = 0
        k = C.c_int()
        while done < n:
            st = self._L.emu_film_ring_submit_many(self._h, C.c_void_p(a[done:].ctypes.data), n - done,
                                                   C.c_void_p(tickets[done:].ctypes.data), C.byref(k))
            for i in range(done, done + k.value):
                self._pending[int(tickets[i])] = (int(a['n_layers'][i]), int(a['n_pw'][i]))
            done += k.value
            if st not in (0, _lib.EMU_E_WORKSPACE):
                check(st, 'emu_film_ring_submit_many')
            if done < n:
                self._drain_some()   # the ring is full until results are read
        return tickets.tolist()

    def _drain_some(self, upto=1024):
        """Read the oldest results that are done (at least the oldest one,
        waiting for it); they free their slots, and poll, poll_many, wait and
        take return them later."""
        oldest = list(itertools.islice(self._pending, upto))
        early = self.poll_many(oldest)
        if not early:
            t = oldest[0]
            early = {t: self._read(t, 60.0)}
        self._early.update(early)

    def poll_many(self, tickets):
        """{ticket: result} for the given tickets that are done (the others
        stay pending), with one call into the library."""
        out, rest = {}, []
        for t in tickets:
            if t in self._early:
                out[t] = self._early.pop(t)
            elif t in self._pending:
                rest.append(t)
            else:
                raise _lib.EmuError(_lib.EMU_E_ARG, 'poll_many: unknown or already read ticket')
        if not rest:
            return out
        if self._RES is None:
            type(self)._RES = self._dtype(_lib.EmuFilmRingResult)
        n = len(rest)
        shp = np.array([self._pending[t] for t in rest], np.int64)
        P, Lm = 2 * shp[:, 1], shp[:, 0] - 1
        ro, lo = np.cumsum(P) - P, np.cumsum(Lm) - Lm
        R, T = np.empty(int(P.sum()), np.complex128), np.empty(int(P.sum()), np.complex128)
        A, Tl = np.empty(int(Lm.sum())), np.empty(int(Lm.sum()))
        Rl, F = np.empty(n), np.empty(n, np.uint32)
        res = np.zeros(n, self._RES)
        idx = np.arange(n)
        res['h_R_net'] = R.ctypes.data + 16 * ro
        res['h_T_net'] = T.ctypes.data + 16 * ro
        res['h_a_list'] = A.ctypes.data + 8 * lo
        res['h_t_list'] = Tl.ctypes.data + 8 * lo
        res['h_r_list'] = Rl.ctypes.data + 8 * idx
        res['h_flags'] = F.ctypes.data + 4 * idx
        done = np.zeros(n, np.int32)
        tk = np.array(rest, np.int64)
        st = self._L.emu_film_ring_poll_many(self._h, C.c_void_p(tk.ctypes.data), n, C.c_void_p(res.ctypes.data),
                                             C.c_void_p(done.ctypes.data))
        if st < 0:
            raise _lib.EmuError(-st, 'emu_film_ring_poll_many')
        for i in np.nonzero(done)[0]:
            t = rest[i]
            del self._pending[t]
            a, b, c, d = ro[i], ro[i] + P[i], lo[i], lo[i] + Lm[i]
            out[t] = {'R_net': R[a:b], 'T_net': T[a:b], 'a_list': A[c:d], 't_list': Tl[c:d],
                      'r_list': Rl[i:i + 1], 'flags': int(F[i])}
        return out

    def _result(self, ticket):
        L, npw = self._pending[ticket]
        res = {'R_net': np.empty(2 * npw, np.complex128), 'T_net': np.empty(2 * npw, np.complex128),
               'a_list': np.empty(L - 1), 't_list': np.empty(L - 1), 'r_list': np.empty(1),
               'flags': np.empty(1, np.uint32)}
        o = _lib.EmuFilmRingResult()
        o.h_R_net, o.h_T_net = (res[k].ctypes.data_as(C.c_void_p) for k in ('R_net', 'T_net'))
        o.h_a_list, o.h_t_list = (res[k].ctypes.data_as(C.c_void_p) for k in ('a_list', 't_list'))
        o.h_r_list, o.h_flags = res['r_list'].ctypes.data_as(C.c_void_p), res['flags'].ctypes.data_as(C.c_void_p)
        return res, o

    def poll(self, ticket):
        if ticket in self._early:
            return self._early.pop(ticket)
        if ticket not in self._pending:
            raise _lib.EmuError(_lib.EMU_E_ARG, 'emu_film_ring_poll: unknown or already read ticket')
        st = self._L.emu_film_ring_ready(self._h, int(ticket))
        if st == 0:
            return None
        if st != 1:
            raise _lib.EmuError(abs(st), 'emu_film_ring_ready')
        return self._read(ticket, 0.0)

    def wait(self, ticket, timeout_s=60.0):
        if ticket in self._early:
            return self._early.pop(ticket)
        if ticket not in self._pending:
            raise _lib.EmuError(_lib.EMU_E_ARG, 'emu_film_ring_wait: unknown or already read ticket')
        return self._read(ticket, timeout_s)

    def _read(self, ticket, timeout_s):
        res, o = self._result(ticket)
        st = self._L.emu_film_ring_wait(self._h, int(ticket), float(timeout_s), C.byref(o))
        if st != 1:
            raise _lib.EmuError(abs(st), 'emu_film_ring_wait')
        del self._pending[ticket]
        res['flags'] = int(res['flags'][0])
        return res

    def _drain_one(self):
        """Read the oldest pending result (it frees its slot); poll, wait
        and take return it later."""
        t = next(iter(self._pending))               # tickets increase: the oldest, O(1)
        self._early[t] = self._read(t, 60.0)

    def take(self, ticket):
        """Result of a ticket, waiting for it if needed (also when it was
        read early to free its slot)."""
        return self.wait(ticket)

    def running(self):
        return bool(self._L.emu_film_ring_running(self._h))

    def stop(self):
        """End the loop; returns the status (EMU_OK, or EMU_E_TIMEOUT if a
        device wait gave up)."""
        return self._L.emu_film_ring_stop(self._h)

    def close(self):
        if self._h is not None:
            self._L.emu_film_ring_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
