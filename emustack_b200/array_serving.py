"""Array-stack requests for the GSM server and the device cache of layer
scattering matrices.

An array stack is one spectral point of a Stack whose layers are a film
substrate, any mix of films and nanostructured (periodic array) layers, and a
film superstrate -- what the reference solves with
``Stack([Anallo, Simmo, ..., Anallo]).calc_scat(pol)`` (backend/stack.py:
162-426).  A nanostructured layer enters as an ``ArrayLayer``: the Bloch
modes a reference Simmo holds after its FEM mode solve (J, J_dag, k_z), or
its air-interface matrices directly.

The interface of a layer with the air reference (R12, T12, R21, T21 of
backend/mode_calcs.py:480-515) is the costly part of a layer and does not
depend on the layer's height or on the other layers of the stack.  The
reference memoises it per (air, layer) object pair
(``_interfaces_i_have_known``, backend/mode_calcs.py:32, 416-448); here it is
kept on the device in ``SMatrixCache`` (LRU, bounded in bytes), so requests
that reuse a layer -- thickness sweeps, stacks that share layers, repeated
queries -- pay only for the cascade.

``ArrayBatcher.launch`` runs one batch of array requests of one shape (order
set, polarisation, layer kinds and Bloch-mode counts) on a stream without
host synchronisation:
  1. host-to-device copy of the packed per-point inputs (pinned staging);
  2. air reference and film k_z for every point (``emu_anallo_modes``,
     batched), film interfaces (``emu_film_interface_batch``);
  3. interfaces of array layers missing from the cache
     (``emu_interface_dense_batch``, batched over the misses of one shape),
     inserted into the cache;
  4. per-position gather of the cached matrices (a layer shared by the whole
     batch is passed once, with a zero batch stride), per-point heights;
  5. cascade + fluxes (``emu_stack_dense_batch``);
  6. device-to-host copy of the outputs into pinned buffers.
"""
from __future__ import annotations

import collections
import ctypes as C
import itertools
import threading

import numpy as np
import torch

from . import _lib
from ._lib import EmuAnalloModes, check, lib, ptr, stream_ptr
from .dense import DenseLayer, DenseStackSolver, film_interface, interface_dense
from .films import grating_orders

c128 = torch.complex128
_LAYER_IDS = itertools.count(1)
_NPW = {}


def _npw(max_order, period, period_y, world_1d):
    key = (max_order, period, period_y, world_1d)
    n = _NPW.get(key)
    if n is None:
        n = _NPW[key] = len(grating_orders(max_order, period, period_y, world_1d)[0])
    return n


def _host_c128(x, shape, name):
    if torch.is_tensor(x):
        if x.dtype != c128 or tuple(x.shape) != shape:
            raise ValueError('%s must be complex128 %s' % (name, shape))
        return x.contiguous()
    a = np.ascontiguousarray(np.asarray(x, dtype=np.complex128))
    if a.shape != shape:
        raise ValueError('%s must have shape %s, got %s' % (name, shape, a.shape))
    t = torch.from_numpy(a)
    return t.pin_memory() if torch.cuda.is_available() else t


class ArrayLayer(object):
    """One nanostructured layer at one spectral point.

    k_z [M]: Bloch-mode propagation constants (normalised like the
    reference's Simmo.k_z).  Then either
      J [P, M] (already divided by the area ratio, backend/mode_calcs.py:
      384-386) and J_dag [M, P]: the interface with the air reference is
      computed on the device on first use (r_t_mat_tf_ns,
      backend/mode_calcs.py:480-515); or
      rt = (R12 [P, P], T12 [M, P], R21 [M, M], T21 [P, M]): the interface
      itself (what the reference's r_t_mat returns).
    Arrays may be host arrays (pinned here for the upload) or CUDA tensors.
    The layer is bound to the spectral point its modes were solved for; a
    request must use it at that point.
    """

    __slots__ = ('key', 'k_z', 'J', 'J_dag', 'rt', 'P', 'M')

    def __init__(self, k_z, J=None, J_dag=None, rt=None):
        kz = np.asarray(k_z.cpu() if torch.is_tensor(k_z) else k_z, dtype=np.complex128).reshape(-1)
        self.M = M = int(kz.shape[0])
        self.k_z = _host_c128(kz, (M,), 'k_z')
        self.key = next(_LAYER_IDS)
        self.J = self.J_dag = self.rt = None
        if (J is None) == (rt is None):
            raise ValueError('ArrayLayer needs either J and J_dag or rt')
        if J is not None:
            if J_dag is None:
                raise ValueError('ArrayLayer needs J_dag with J')
            P = int(J.shape[0])
            self.J = _host_c128(J, (P, M), 'J')
            self.J_dag = _host_c128(J_dag, (M, P), 'J_dag')
        else:
            R12, T12, R21, T21 = rt
            P = int(R12.shape[0])
            self.rt = (_host_c128(R12, (P, P), 'R12'), _host_c128(T12, (M, P), 'T12'),
                       _host_c128(R21, (M, M), 'R21'), _host_c128(T21, (P, M), 'T21'))
        self.P = P

    def smatrix_bytes(self):
        """Device bytes of its cached interface and k_z."""
        P, M = self.P, self.M
        return 16 * (P * P + 2 * M * P + M * M + M) + 4


class ArrayRequest(object):
    """One spectral point of an array stack.

    layers: bottom (substrate) to top (superstrate); the first and the last
    are film indices (complex, loss applied), the others film indices or
    ``ArrayLayer``s.  heights_nm: the finite layers' heights (len(layers) - 2).
    wl_nm, k_pll [2] (nm^-1), period, max_order (the Light's max_order_PWs),
    period_y, world_1d as for the reference's Light / ThinFilm / NanoStruct;
    pol a polarisation name, or incoming [2 Npw] amplitudes on the
    superstrate (backend/stack.py:162-186).
    """

    __slots__ = ('layers', 'heights', 'wl_nm', 'k_pll', 'period', 'period_y', 'max_order',
                 'world_1d', 'pol', 'incoming', 'npw', 'signature', 'air_key', 't_submit',
                 't_arrival', 'future', '_nbytes')

    def __init__(self, layers, heights_nm, wl_nm, k_pll, period, max_order, pol='TE',
                 period_y=None, world_1d=False, incoming=None, t_arrival=None):
        if len(layers) < 2:
            raise ValueError('a stack needs at least a substrate and a superstrate')
        if isinstance(layers[0], ArrayLayer) or isinstance(layers[-1], ArrayLayer):
            raise NotImplementedError('array requests need film substrate and superstrate')
        self.period = float(period)
        self.period_y = float(period if period_y is None else period_y)
        self.max_order = int(max_order)
        self.world_1d = bool(world_1d)
        self.npw = _npw(self.max_order, self.period, self.period_y, self.world_1d)
        P = 2 * self.npw
        self.layers = []
        kinds = []
        for i, ly in enumerate(layers):
            if isinstance(ly, ArrayLayer):
                if ly.P != P:
                    raise ValueError("Scattering matrices of layers are not consistent: layer %d has "
                                     "%d plane waves, the order set %d" % (i, ly.P, P))
                self.layers.append(ly)
                kinds.append(ly.M)
            else:
                self.layers.append(complex(ly))
                kinds.append(0)
        self.heights = np.asarray(heights_nm, dtype=np.float64).reshape(-1)
        if self.heights.shape[0] != len(layers) - 2:
            raise ValueError('need one height per finite layer')
        self.wl_nm = float(wl_nm)
        self.k_pll = np.asarray(k_pll, dtype=np.float64).reshape(2)
        if incoming is not None:
            self.incoming = np.asarray(incoming, dtype=np.complex128).reshape(-1)
            if self.incoming.shape[0] != P:
                raise ValueError('incoming must have 2 Npw = %d amplitudes' % P)
            self.pol = 'incoming'
        else:
            if pol not in _lib.POL:
                raise NotImplementedError('Must select from the currently implemented polarisations; '
                                          'TE, TM, R Circ, L Circ.')
            self.incoming = None
            self.pol = pol
        self.signature = ('array', self.max_order, self.period, self.period_y, self.world_1d,
                          self.pol, tuple(kinds))
        self.air_key = (self.wl_nm, float(self.k_pll[0]), float(self.k_pll[1]), self.max_order,
                        self.period, self.period_y, self.world_1d)
        self.t_arrival = t_arrival
        self._nbytes = None

    def max_dim(self):
        """D = max(P, M of every array layer): the size of the cascade's matrices."""
        return max([2 * self.npw] + [ly.M for ly in self.layers if isinstance(ly, ArrayLayer)])

    def wl_norm(self):
        """wl / period, nudged off exact multiples (backend/mode_calcs.py:45-49)."""
        w = self.wl_nm / self.period
        if self.wl_nm % self.period == 0:
            w += 1e-10
        return w

    def bytes_on_device(self):
        """Device bytes of this point inside its batch (gathered layer
        matrices, film interfaces, cascade workspace, outputs); the cached
        interfaces themselves are counted by the cache."""
        if self._nbytes is None:
            P = 2 * self.npw
            Ms = [ly.M if isinstance(ly, ArrayLayer) else P for ly in self.layers]
            dense = [isinstance(ly, ArrayLayer) for ly in self.layers]
            nb = 0
            for M, d in zip(Ms, dense):
                nb += 16 * (P * P + 2 * M * P + M * M + M) if d else 16 * (4 * P + P)
            nb += dense_workspace_bytes(P, Ms)
            nb += 16 * (2 * P * P) + 16 * (3 * len(Ms)) + 8 * len(Ms) + 512
            self._nbytes = nb
        return self._nbytes


def dense_workspace_bytes(P, Ms):
    """Per-point workspace of emu_stack_dense_batch for layer sizes Ms
    (the library's emu_stack_dense_workspace_size for a batch of one, without
    the fixed 256 bytes)."""
    L = len(Ms)
    D = max([P] + list(Ms))
    Lf = L - 2 if L > 2 else 0
    elems = (2 * L - 2 + L - 1 + Lf + 4) * D * D + Lf * D + 6 * D
    return elems * 16 + ((D * 4 + 15) // 16) * 16


class _Entry(object):
    """Cached interface of one array layer with one air reference."""

    __slots__ = ('R12', 'T12', 'R21', 'T21', 'kz', 'info', 'ready', 'users', 'nbytes', 'bad')

    def __init__(self, R12, T12, R21, T21, kz, info, ready, nbytes):
        self.R12, self.T12, self.R21, self.T21 = R12, T12, R21, T21
        self.kz, self.info, self.ready = kz, info, ready
        self.users = 0
        self.nbytes = nbytes
        self.bad = False


class SMatrixCache(object):
    """Device-resident layer interfaces, least recently used first out.

    capacity_bytes bounds the bytes held; entries in use by batches in flight
    (``users`` > 0) are not evicted, so the cache can exceed its capacity
    until those batches finish.  Keys are (layer key, air key).
    """

    def __init__(self, capacity_bytes):
        self.capacity = int(capacity_bytes)
        self.entries = collections.OrderedDict()
        self.bytes = 0
        self.hits = self.misses = self.evictions = 0

    def get(self, key):
        e = self.entries.get(key)
        if e is None:
            self.misses += 1
        else:
            self.hits += 1
            self.entries.move_to_end(key)
        return e

    def put(self, key, entry):
        old = self.entries.pop(key, None)
        if old is not None:
            self.bytes -= old.nbytes
        self.entries[key] = entry
        self.bytes += entry.nbytes
        self.evict()

    def drop(self, key):
        e = self.entries.pop(key, None)
        if e is not None:
            self.bytes -= e.nbytes

    def evict(self):
        if self.bytes <= self.capacity:
            return
        for key in list(self.entries):
            if self.bytes <= self.capacity:
                break
            e = self.entries[key]
            if e.users:
                continue
            del self.entries[key]
            self.bytes -= e.nbytes
            self.evictions += 1

    def stats(self):
        n = self.hits + self.misses
        return dict(entries=len(self.entries), bytes=self.bytes, hits=self.hits, misses=self.misses,
                    evictions=self.evictions, hit_rate=self.hits / n if n else float('nan'))


def _pinned(shape, dtype):
    return torch.empty(shape, dtype=dtype).pin_memory()


class ArrayBatcher(object):
    """Runs batches of array requests of one signature on a stream."""

    def __init__(self, device, cache):
        self.device = device
        self.cache = cache
        # the cache and the entries' use counts are shared by batches launched
        # from several threads
        self.lock = threading.Lock()
        self._orders = {}
        self._solvers = {}

    def _order_tensors(self, r):
        key = (r.max_order, r.period, r.period_y, r.world_1d)
        t = self._orders.get(key)
        if t is None:
            px, py = grating_orders(*key)
            t = self._orders[key] = (torch.from_numpy(px).to(self.device),
                                     torch.from_numpy(py).to(self.device))
        return t

    def _modes(self, r, px, py, wl, kp, n, sort_in):
        """Sorted film k_z of every point (backend/mode_calcs.py:116-186)."""
        B, npw = int(wl.shape[0]), r.npw
        kz = torch.empty((B, npw), dtype=c128, device=self.device)
        sort_out = torch.empty((B, npw), dtype=torch.int32, device=self.device)
        spec = torch.empty(B, dtype=torch.int32, device=self.device)
        nprop = torch.empty(B, dtype=torch.int32, device=self.device)
        d = EmuAnalloModes()
        d.n_points, d.n_pw, d.world_1d = B, npw, int(r.world_1d)
        d.period, d.period_y = r.period, r.period_y
        d.d_px, d.d_py = ptr(px), ptr(py)
        d.d_wl_nm, d.d_k_pll, d.d_n = ptr(wl), ptr(kp), ptr(n)
        d.d_sort_in = ptr(sort_in)
        d.d_kz, d.d_sort_out, d.d_specular, d.d_num_prop = ptr(kz), ptr(sort_out), ptr(spec), ptr(nprop)
        check(lib().emu_anallo_modes(C.byref(d), stream_ptr()), 'emu_anallo_modes')
        return kz, sort_out, spec, nprop

    def _fill(self, reqs, pos_of, air_of, stream, pins=None):
        """Cache entries of the array layers of every request; computes and
        inserts the missing ones.  pos_of(b) lists request b's array
        positions; air_of(b) = (kz_air, wln, row) locates its air reference
        in the device tensors of its order set.  Returns {(b, pos): cache
        key} and the distinct entries used {key: entry}."""
        with self.lock:
            key_at, used = self._fill_locked(reqs, pos_of, air_of, stream)
            if pins is not None:
                pins.extend(used.values())
            return key_at, used

    def _unpin(self, pins):
        """Release the entries a batch pinned when its launch failed."""
        with self.lock:
            for e in pins:
                e.users -= 1
            self.cache.evict()

    def _fill_locked(self, reqs, pos_of, air_of, stream):
        cache = self.cache
        key_at = {}
        used = {}
        missing = collections.OrderedDict()   # cache key -> (layer, request index)
        for b, r in enumerate(reqs):
            for j in pos_of(b):
                ly = r.layers[j]
                key = (ly.key, r.air_key)
                if key not in used and key not in missing:
                    e = cache.get(key)
                    if e is None:
                        missing[key] = (ly, b)
                    else:
                        used[key] = e
                key_at[(b, j)] = key
        # compute the misses, batched by (source, P, M, air tensors)
        groups = collections.defaultdict(list)
        for key, (ly, b) in missing.items():
            kz_air, wln, _ = air_of(b)
            groups[(ly.J is not None, ly.P, ly.M, id(kz_air))].append((key, ly, b))
        for (from_J, _, M, _), items in groups.items():
            nm = len(items)
            kz = self._upload([ly.k_z for _, ly, _ in items])
            if from_J:
                J = self._upload([ly.J for _, ly, _ in items])
                Jd = self._upload([ly.J_dag for _, ly, _ in items])
                kz_air, wln, _ = air_of(items[0][2])
                idx = torch.tensor([air_of(b)[2] for _, _, b in items], dtype=torch.long, device=self.device)
                R12, T12, R21, T21, info = interface_dense(
                    kz_air.index_select(0, idx).contiguous(), torch.ones(nm, dtype=c128, device=self.device),
                    wln.index_select(0, idx).contiguous(), J, Jd)
            else:
                R12, T12, R21, T21 = (self._upload([ly.rt[k] for _, ly, _ in items]) for k in range(4))
                info = torch.zeros(nm, dtype=torch.int32, device=self.device)
            entries = []
            for i, (key, ly, _) in enumerate(items):
                e = _Entry(R12[i:i + 1].clone(), T12[i:i + 1].clone(), R21[i:i + 1].clone(),
                           T21[i:i + 1].clone(), kz[i:i + 1].clone(), info[i:i + 1].clone(), None,
                           ly.smatrix_bytes())
                used[key] = e
                entries.append(e)
            ev = torch.cuda.Event()
            ev.record(stream)          # after the copies into the entries
            for e in entries:
                e.ready = ev
        for e in used.values():        # pinned until this batch finishes
            e.users += 1
        for key in missing:
            cache.put(key, used[key])
        for e in used.values():
            stream.wait_event(e.ready)
        return key_at, used

    def _upload(self, ts):
        """Stack host (pinned) or device tensors of one shape on the device,
        asynchronously on the current stream."""
        out = torch.empty((len(ts),) + tuple(ts[0].shape), dtype=ts[0].dtype, device=self.device)
        for i, t in enumerate(ts):
            out[i].copy_(t, non_blocking=True)
        return out

    def launch(self, reqs, stream, slot_key):
        """Queue one batch of array requests of one signature on ``stream``;
        returns (event, finish) where finish() -> list of per-request results
        (dicts) or exceptions.  A launch that fails releases the cache
        entries it pinned before raising."""
        pins = []
        try:
            return self._launch_grouped(reqs, stream, slot_key, pins)
        except Exception:
            self._unpin(pins)
            raise

    def _launch_grouped(self, reqs, stream, slot_key, pins):
        r0 = reqs[0]
        B, npw = len(reqs), r0.npw
        P = 2 * npw
        dev = self.device
        L = len(r0.layers)
        film_pos = [j for j, ly in enumerate(r0.layers) if not isinstance(ly, ArrayLayer)]
        arr_pos = [j for j, ly in enumerate(r0.layers) if isinstance(ly, ArrayLayer)]
        # packed host inputs
        h_wl = _pinned((B,), torch.float64)
        h_kp = _pinned((B, 2), torch.float64)
        h_wln = _pinned((B,), torch.float64)
        h_n = _pinned((len(film_pos), B), c128)
        h_h = _pinned((max(L - 2, 1), B), torch.float64)
        h_wl.numpy()[:] = [r.wl_nm for r in reqs]
        h_kp.numpy()[:] = np.stack([r.k_pll for r in reqs])
        h_wln.numpy()[:] = [r.wl_norm() for r in reqs]
        h_n.numpy()[:] = np.array([[r.layers[j] for r in reqs] for j in film_pos], dtype=np.complex128)
        if L > 2:
            h_h.numpy()[:] = np.stack([r.heights for r in reqs], axis=1) / r0.period
        h_inc = None
        if r0.incoming is not None:
            h_inc = _pinned((B, P), c128)
            h_inc.numpy()[:] = np.stack([r.incoming for r in reqs])
        px, py = self._order_tensors(r0)
        with torch.cuda.stream(stream):
            wl = h_wl.to(dev, non_blocking=True)
            kp = h_kp.to(dev, non_blocking=True)
            wln = h_wln.to(dev, non_blocking=True)
            nfilm = h_n.to(dev, non_blocking=True)
            hn = h_h.to(dev, non_blocking=True)
            inc = h_inc.to(dev, non_blocking=True) if h_inc is not None else None
            n_air = torch.ones(B, dtype=c128, device=dev)
            kz_air, sort_air, spec, np_air = self._modes(r0, px, py, wl, kp, n_air, None)
            layers = [None] * L
            np_top = np_sub = None
            for f, j in enumerate(film_pos):
                nj = nfilm[f]
                kz, _, _, npj = self._modes(r0, px, py, wl, kp, nj, sort_air)
                R, T = film_interface(kz_air, n_air, kz, nj, wln)
                fin = 0 < j < L - 1
                layers[j] = DenseLayer(R, T, torch.neg(R), T, False,
                                       torch.cat([kz, kz], dim=1) if fin else None,
                                       hn[j - 1] if fin else 0.0)
                if j == 0:
                    np_sub = npj
                if j == L - 1:
                    np_top = npj
            key_at, used = self._fill(reqs, lambda b: arr_pos, lambda b: (kz_air, wln, b), stream, pins)
            for j in arr_pos:
                keys = [key_at[(b, j)] for b in range(B)]
                es = [used[k] for k in keys]
                if all(k == keys[0] for k in keys):
                    e = es[0]
                    R12, T12, R21, T21, kz = e.R12, e.T12, e.R21, e.T21, e.kz
                else:
                    R12, T12, R21, T21, kz = (torch.cat([getattr(e, nm) for e in es])
                                              for nm in ('R12', 'T12', 'R21', 'T21', 'kz'))
                layers[j] = DenseLayer(R12, T12, R21, T21, True, kz, hn[j - 1])
            nprop = torch.stack([np_air, np_top, np_sub], dim=1).contiguous()
            solver = self._solvers.get(slot_key)
            if solver is None:
                solver = self._solvers[slot_key] = DenseStackSolver(dev)
            out = solver.solve(layers, P, pol=r0.pol if inc is None else 'TE', incoming=inc,
                               specular=spec, num_prop=nprop)
            ukeys = list(used)
            infos = torch.cat([used[k].info for k in ukeys]) if ukeys else None
            host = {}
            for k in ('R_net', 'T_net', 'a_list', 't_list', 'r_list', 'flags', 'info'):
                t = _pinned(tuple(out[k].shape), out[k].dtype)
                t.copy_(out[k], non_blocking=True)
                host[k] = t
            if infos is not None:
                host['layer_info'] = _pinned(tuple(infos.shape), infos.dtype)
                host['layer_info'].copy_(infos, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(stream)

        def result(h, b):
            return {'R_net': h['R_net'][b], 'T_net': h['T_net'][b], 'a_list': h['a_list'][b],
                    't_list': h['t_list'][b], 'r_list': float(h['r_list'][b]), 'flags': int(h['flags'][b])}

        return ev, self._finisher(reqs, host, ukeys, used, key_at, result)

    def _finisher(self, reqs, host, ukeys, used, key_at, result):
        """finish(): releases the batch's cache entries (dropping singular
        ones) and returns each request's result or exception."""
        cache = self.cache

        lock = self.lock

        def finish():
            h = {k: v.numpy() for k, v in host.items()}
            bad = set()
            with lock:
                for i, k in enumerate(ukeys):
                    e = used[k]
                    e.users -= 1
                    if int(h['layer_info'][i]) != 0:
                        e.bad = True
                        bad.add(k)
                        cache.drop(k)
                cache.evict()
            res = []
            for b, r in enumerate(reqs):
                if int(h['info'][b]) != 0 or any(k in bad for (bb, _), k in key_at.items() if bb == b):
                    res.append(np.linalg.LinAlgError('Singular matrix'))
                elif int(h['flags'][b]) & _lib.PT_BAD_POINT:
                    res.append(_lib.EmuError(_lib.EMU_E_SHAPE, 'array request'))
                else:
                    res.append(result(h, b))
            return res

        return finish

    def launch_uneven(self, reqs, stream, slot_key, ws_budget_bytes):
        """Array requests of any shapes as one uneven batch (see
        _launch_uneven); releases its pinned cache entries if it fails."""
        pins = []
        try:
            return self._launch_uneven(reqs, stream, slot_key, ws_budget_bytes, pins)
        except Exception:
            self._unpin(pins)
            raise

    def _launch_uneven(self, reqs, stream, slot_key, ws_budget_bytes, pins):
        """Queues array requests of ANY shapes as one uneven batch on
        ``stream``: film modes and interfaces per order set, cached array
        interfaces, then one emu_stack_var_batch launch for every cascade.
        Returns (event, finish) as ``launch``."""
        from .dense import StackVarSolver, VarStack
        dev = self.device
        sets = collections.OrderedDict()
        for b, r in enumerate(reqs):
            sets.setdefault((r.max_order, r.period, r.period_y, r.world_1d), []).append(b)
        n = len(reqs)
        air = [None] * n                 # (kz_air, wln, row) per request
        film_of = [None] * n             # (R, T, -R, kz2) of the request's order set
        film = {}                        # (b, j) -> row of the film instance in those tensors
        np_parts, spec_parts, order = [], [], []
        keep = []
        with torch.cuda.stream(stream):
            for key, bs in sets.items():
                r0 = reqs[bs[0]]
                B = len(bs)
                inst = [(b, j) for b in bs for j, ly in enumerate(reqs[b].layers)
                        if not isinstance(ly, ArrayLayer)]
                rows = {b: i for i, b in enumerate(bs)}
                h = _pinned((4 * B + 4 * len(inst),), torch.float64)
                hv = h.numpy()
                hv[0:B] = [reqs[b].wl_nm for b in bs]
                hv[B:3 * B] = np.stack([reqs[b].k_pll for b in bs]).reshape(-1)
                hv[3 * B:4 * B] = [reqs[b].wl_norm() for b in bs]
                o = 4 * B
                hv[o:o + 2 * len(inst)].view(np.complex128)[:] = [reqs[b].layers[j] for b, j in inst]
                hv[o + 2 * len(inst):o + 4 * len(inst)] = [rows[b] for b, _ in inst] + [0] * len(inst)
                d = h.to(dev, non_blocking=True)
                keep.append(h)
                wl, kp, wln = d[0:B], d[B:3 * B].view(B, 2), d[3 * B:4 * B]
                nf = d[o:o + 2 * len(inst)].view(c128)
                irow = d[o + 2 * len(inst):o + 3 * len(inst)].to(torch.long)
                px, py = self._order_tensors(r0)
                n_air = torch.ones(B, dtype=c128, device=dev)
                kz_air, sort_air, spec, np_air = self._modes(r0, px, py, wl, kp, n_air, None)
                kz_i = kz_air.index_select(0, irow)
                kz_f, _, _, np_f = self._modes(r0, px, py, wl.index_select(0, irow),
                                               kp.index_select(0, irow).contiguous(), nf,
                                               sort_air.index_select(0, irow).contiguous())
                R, T = film_interface(kz_i, torch.ones(len(inst), dtype=c128, device=dev), kz_f, nf,
                                      wln.index_select(0, irow))
                mR = torch.neg(R)
                kz2 = torch.cat([kz_f, kz_f], dim=1)
                keep += [R, T, mR, kz2]
                top = {}
                sub = {}
                for i, (b, j) in enumerate(inst):
                    film[(b, j)] = i
                    if j == 0:
                        sub[b] = i
                    if j == len(reqs[b].layers) - 1:
                        top[b] = i
                for b in bs:
                    air[b] = (kz_air, wln, rows[b])
                    film_of[b] = (R, T, mR, kz2)
                ti = torch.tensor([top[b] for b in bs], dtype=torch.long, device=dev)
                si = torch.tensor([sub[b] for b in bs], dtype=torch.long, device=dev)
                np_parts.append(torch.stack([np_air, np_f.index_select(0, ti), np_f.index_select(0, si)], 1))
                spec_parts.append(spec)
                order += bs
            key_at, used = self._fill(
                reqs, lambda b: [j for j, ly in enumerate(reqs[b].layers) if isinstance(ly, ArrayLayer)],
                lambda b: air[b], stream, pins)
            stacks = []
            inc_keep = []
            for b in order:
                r = reqs[b]
                P, L = 2 * r.npw, len(r.layers)
                R, T, mR, kz2 = film_of[b]
                lays = []
                for j, ly in enumerate(r.layers):
                    fin = 0 < j < L - 1
                    hn = float(r.heights[j - 1]) / r.period if fin else 0.0
                    if isinstance(ly, ArrayLayer):
                        e = used[key_at[(b, j)]]
                        lays.append((e.R12[0], e.T12[0], e.R21[0], e.T21[0], True, e.kz[0], hn))
                    else:
                        i = film[(b, j)]
                        lays.append((R[i], T[i], mR[i], T[i], False, kz2[i] if fin else None, hn))
                inc = None
                if r.incoming is not None:
                    hi = _pinned((P,), c128)
                    hi.numpy()[:] = r.incoming
                    inc = hi.to(dev, non_blocking=True)
                    inc_keep.append(hi)
                stacks.append(VarStack(lays, P, pol=r.pol if inc is None else 'TE', incoming=inc))
            solver = self._solvers.get(('uneven', slot_key))   # one workspace per stream
            if solver is None:
                solver = self._solvers[('uneven', slot_key)] = StackVarSolver(dev)
            out = solver.solve(stacks, spec=torch.cat(spec_parts), num_prop=torch.cat(np_parts),
                               ws_budget_bytes=ws_budget_bytes)
            ukeys = list(used)
            host = {}
            for k in ('R_net', 'T_net', 'a_list', 't_list', 'r_list', 'flags', 'info'):
                t = _pinned(tuple(out[k].shape), out[k].dtype)
                t.copy_(out[k], non_blocking=True)
                host[k] = t
            if ukeys:
                infos = torch.cat([used[k].info for k in ukeys])
                host['layer_info'] = _pinned(tuple(infos.shape), infos.dtype)
                host['layer_info'].copy_(infos, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(stream)
        # results come back in `order`; map them to the requests' positions
        pos = {b: i for i, b in enumerate(order)}
        ro, lo = out['rnet_off'], out['list_off']
        ordered = [reqs[b] for b in order]
        key_at_o = {(pos[b], j): k for (b, j), k in key_at.items()}

        def result(h, i):
            r = ordered[i]
            P, L = 2 * r.npw, len(r.layers)
            a, c = int(ro[i]), int(lo[i])
            return {'R_net': h['R_net'][a:a + P * P].reshape(P, P), 'T_net': h['T_net'][a:a + P * P].reshape(P, P),
                    'a_list': h['a_list'][c:c + L - 1], 't_list': h['t_list'][c:c + L - 1],
                    'r_list': float(h['r_list'][i]), 'flags': int(h['flags'][i])}

        fin_o = self._finisher(ordered, host, ukeys, used, key_at_o, result)
        keep.append(out)

        def finish():
            res_o = fin_o()
            keep.clear()
            inc_keep.clear()
            return [res_o[pos[b]] for b in range(n)]

        return ev, finish
