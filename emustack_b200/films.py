"""Batched all-film stacks on the GPU (one fused launch per batch).

A stack whose every layer is a homogeneous film (reference: ``Anallo``) has
only diagonal interface, propagation and cascade matrices
(backend/mode_calcs.py:451-477, backend/stack.py:162-426).  This module
solves a batch of such spectral points through ``emu_film_stack_batch``:
device-resident inputs in, device-resident R_net / T_net diagonals,
a_list / t_list / r_list and (optionally) every intermediate the reference
exposes out.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import EmuFilmStackBatch, check, lib, ptr, stream_ptr


def grating_orders(max_order, period, period_y=None, world_1d=False):
    """Plane-wave orders (px, py) in the reference's order (mode_calcs.py:55-74)."""
    period_y = period if period_y is None else period_y
    L = lib()
    n = C.c_int(0)
    check(L.emu_grating_orders(int(max_order), float(period), float(period_y), int(bool(world_1d)),
                               None, None, 0, C.byref(n)), 'emu_grating_orders')
    px = np.zeros(n.value, np.int32)
    py = np.zeros(n.value, np.int32)
    check(L.emu_grating_orders(int(max_order), float(period), float(period_y), int(bool(world_1d)),
                               px.ctypes.data_as(C.c_void_p), py.ctypes.data_as(C.c_void_p),
                               n.value, C.byref(n)), 'emu_grating_orders')
    return px, py


OPTIONAL = ('kz', 'layer_rt', 'vec_coef', 'fluxes', 'sort_order', 'specular', 'num_prop')


class FilmStackSolver(object):
    """Reusable device buffers for batches of all-film stacks.

    Parameters mirror the reference objects: ``period``/``period_y`` of the
    ThinFilms, ``max_order`` of the Light (``max_order_PWs``), ``world_1d``.
    """

    def __init__(self, n_layers, max_order, period, period_y=None, world_1d=False,
                 device='cuda'):
        if n_layers < 2:
            raise ValueError('a stack needs at least a substrate and a superstrate')
        self.L = int(n_layers)
        self.period = float(period)
        self.period_y = float(period if period_y is None else period_y)
        self.world_1d = bool(world_1d)
        self.max_order = int(max_order)
        self.device = torch.device(device)
        px, py = grating_orders(max_order, self.period, self.period_y, world_1d)
        self.px_host, self.py_host = px, py
        self.npw = len(px)
        self.P = 2 * self.npw
        self.d_px = torch.from_numpy(px).to(self.device)
        self.d_py = torch.from_numpy(py).to(self.device)
        self._bufs = {}
        self._ws = None

    # ------------------------------------------------------------------
    def _buf(self, name, shape, dtype):
        t = self._bufs.get(name)
        if t is None or tuple(t.shape) != tuple(shape) or t.dtype != dtype:
            t = torch.empty(shape, dtype=dtype, device=self.device)
            self._bufs[name] = t
        return t

    def outputs(self, B, want=()):
        L, P, npw = self.L, self.P, self.npw
        o = {
            'R_net': self._buf('R_net', (B, P), torch.complex128),
            'T_net': self._buf('T_net', (B, P), torch.complex128),
            'a_list': self._buf('a_list', (B, L - 1), torch.float64),
            't_list': self._buf('t_list', (B, L - 1), torch.float64),
            'r_list': self._buf('r_list', (B,), torch.float64),
            'flags': self._buf('flags', (B,), torch.int32),
        }
        if 'kz' in want:
            o['kz'] = self._buf('kz', (B, L, npw), torch.complex128)
        if 'layer_rt' in want:
            o['layer_rt'] = self._buf('layer_rt', (B, L, 2, P), torch.complex128)
        if 'vec_coef' in want:
            o['vec_coef_down'] = self._buf('vcd', (B, L, P), torch.complex128)
            o['vec_coef_up'] = self._buf('vcu', (B, L - 1, P), torch.complex128)
        if 'fluxes' in want:
            o['fluxes'] = self._buf('fluxes', (B, L + 1, 2), torch.float64)
        if 'sort_order' in want:
            o['sort_order'] = self._buf('sort_order', (B, npw), torch.int32)
        if 'specular' in want:
            o['specular'] = self._buf('specular', (B,), torch.int32)
        if 'num_prop' in want:
            o['num_prop'] = self._buf('num_prop', (B, L + 1), torch.int32)
        return o

    def descriptor(self, wl_nm, k_pll, n, heights_nm, pol, incoming, shears, out):
        B = int(wl_nm.shape[0])
        d = EmuFilmStackBatch()
        d.n_points = B
        d.n_layers = self.L
        d.n_pw = self.npw
        d.world_1d = int(self.world_1d)
        d.period = self.period
        d.period_y = self.period_y
        d.d_px = ptr(self.d_px)
        d.d_py = ptr(self.d_py)
        d.d_wl_nm = ptr(wl_nm)
        d.d_k_pll = ptr(k_pll)
        d.d_n = ptr(n)
        d.d_heights_nm = ptr(heights_nm) if heights_nm is not None and heights_nm.numel() else None
        d.heights_per_point = int(heights_nm is not None and heights_nm.dim() == 2)
        if incoming is not None:
            d.pol = _lib.POL_INCOMING
            d.d_incoming = ptr(incoming)
        else:
            if pol not in _lib.POL:
                raise NotImplementedError('Must select from the currently implemented polarisations; '
                                          'TE, TM, R Circ, L Circ.')
            d.pol = _lib.POL[pol]
        if shears is not None:
            d.d_shears = ptr(shears)
            d.shear_ncoord = int(shears.shape[1])
        d.d_R_net = ptr(out['R_net'])
        d.d_T_net = ptr(out['T_net'])
        d.d_a_list = ptr(out['a_list'])
        d.d_t_list = ptr(out['t_list'])
        d.d_r_list = ptr(out['r_list'])
        d.d_flags = ptr(out['flags'])
        d.d_kz = ptr(out.get('kz'))
        d.d_layer_rt = ptr(out.get('layer_rt'))
        d.d_vec_coef_down = ptr(out.get('vec_coef_down'))
        d.d_vec_coef_up = ptr(out.get('vec_coef_up'))
        d.d_fluxes = ptr(out.get('fluxes'))
        d.d_sort_order = ptr(out.get('sort_order'))
        d.d_specular = ptr(out.get('specular'))
        d.d_num_prop = ptr(out.get('num_prop'))
        return d

    def workspace(self, nbytes):
        if self._ws is None or self._ws.numel() < nbytes:
            self._ws = torch.empty(max(int(nbytes), 16), dtype=torch.uint8, device=self.device)
        return self._ws

    def solve(self, wl_nm, k_pll, n, heights_nm=None, pol='TE', incoming=None, shears=None,
              want=(), stream=None, variant=None):
        """Solve a batch on the device.

        wl_nm   float64 [B]           k_pll float64 [B, 2] (nm^-1)
        n       complex128 [B, L]     (loss already applied)
        heights float64 [L-2] or [B, L-2] (nm)
        incoming complex128 [B, P] or None (then ``pol`` selects the
        specular incidence of backend/mode_calcs.py:220-250)
        shears  float64 [L, ncoord] or None
        variant launch variant of the film kernel (``EmuFilmStackBatch.variant``);
                None: the autotuner's choice for this shape (timed on first
                use), results do not depend on it
        Returns a dict of device tensors (reused across calls).
        """
        for t, nm, dt in ((wl_nm, 'wl_nm', torch.float64), (k_pll, 'k_pll', torch.float64),
                          (n, 'n', torch.complex128)):
            if not t.is_cuda or not t.is_contiguous() or t.dtype != dt:
                raise TypeError('%s must be a contiguous CUDA %s tensor' % (nm, dt))
        if heights_nm is not None and (heights_nm.dtype != torch.float64 or not heights_nm.is_cuda
                                       or not heights_nm.is_contiguous()):
            raise TypeError('heights_nm must be a contiguous CUDA float64 tensor')
        if incoming is not None and (incoming.dtype != torch.complex128 or not incoming.is_cuda):
            raise TypeError('incoming must be a CUDA complex128 tensor')
        if shears is not None and (shears.dtype != torch.float64 or not shears.is_cuda):
            raise TypeError('shears must be a CUDA float64 tensor')
        B = int(wl_nm.shape[0])
        if tuple(n.shape) != (B, self.L) or n.dtype != torch.complex128:
            raise ValueError('n must be complex128 [B, L]')
        if tuple(k_pll.shape) != (B, 2):
            raise ValueError('k_pll must be float64 [B, 2]')
        out = self.outputs(B, want)
        d = self.descriptor(wl_nm, k_pll, n, heights_nm, pol, incoming, shears, out)
        L = lib()
        nbytes = L.emu_film_stack_workspace_size(C.byref(d))
        ws = self.workspace(nbytes)

        def run(v):
            d.variant = int(v)
            check(L.emu_film_stack_batch(C.byref(d), ptr(ws), C.c_size_t(ws.numel()),
                                         stream_ptr(stream)), 'emu_film_stack_batch')

        if variant is None:
            from .autotune import default_tuner, size_bucket
            shape = dict(L=self.L, npw=self.npw, B=size_bucket(B), inc=incoming is not None,
                         opt=sorted(want))
            variant = default_tuner().choose('film_stack', shape, list(_lib.FILM_VARIANTS), run, 0,
                                             stream=stream)
        run(variant)
        return out


class FilmHostPipeline(object):
    """Host-to-host solves of batches of all-film stacks of one shape.

    Inputs come from (pinned) host tensors and results land in pinned host
    tensors.  The batch is cut into `chunk`-point pieces dealt round-robin to
    `n_streams` streams, each with its own FilmStackSolver, so the
    device-to-host copy of one piece's R_net / T_net / lists overlaps the
    solve of the next and the host-to-device copy of the one after: the
    host link and the SMs work at the same time.  Arguments as
    FilmStackSolver; results as its `solve` (the same kernel per point).
    """

    OUT = ('R_net', 'T_net', 'a_list', 't_list', 'r_list', 'flags')
    SPECTRA = ('a_list', 't_list', 'r_list', 'flags')

    def __init__(self, n_layers, max_order, period, period_y=None, world_1d=False, device='cuda',
                 chunk=8192, n_streams=2, outputs=OUT):
        """outputs: the results copied back to the host, a subset of OUT
        (SPECTRA: the absorptance / transmittance / reflectance lists and
        flags only, the R/T/A spectra of a sweep; R_net and T_net are
        computed on the device either way)."""
        if not outputs or any(k not in self.OUT for k in outputs):
            raise ValueError('outputs must be a non-empty subset of %s' % (self.OUT,))
        self.keys = tuple(outputs)
        self.device = torch.device(device)
        self.solvers = [FilmStackSolver(n_layers, max_order, period, period_y, world_1d, device=self.device)
                        for _ in range(n_streams)]
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(n_streams)]
        self.chunk = int(chunk)
        self._out = None

    def outputs(self, B):
        """Pinned host outputs for a batch of B points (reused across calls)."""
        if self._out is None or next(iter(self._out.values())).shape[0] != B:
            dev = self.solvers[0].outputs(1)
            self._out = {k: torch.empty((B,) + tuple(dev[k].shape[1:]), dtype=dev[k].dtype).pin_memory()
                         for k in self.keys}
        return self._out

    def solve(self, wl_nm, k_pll, n, heights_nm=None, pol='TE', variant=None):
        """wl_nm float64 [B], k_pll float64 [B, 2], n complex128 [B, L],
        heights_nm float64 [L-2] or [B, L-2]: host tensors (pinned for
        asynchronous copies).  Returns the pinned host outputs; the current
        stream waits for every piece, so they are complete once it has
        reached this point (e.g. after torch.cuda.synchronize())."""
        B = int(wl_nm.shape[0])
        out = self.outputs(B)
        cur = torch.cuda.current_stream(self.device)
        for st in self.streams:
            st.wait_stream(cur)
        per_point_h = heights_nm is not None and heights_nm.dim() == 2
        for c, b0 in enumerate(range(0, B, self.chunk)):
            b1 = min(B, b0 + self.chunk)
            i = c % len(self.streams)
            st, sol = self.streams[i], self.solvers[i]
            with torch.cuda.stream(st):
                dw = wl_nm[b0:b1].to(self.device, non_blocking=True)
                dk = k_pll[b0:b1].to(self.device, non_blocking=True)
                dn = n[b0:b1].to(self.device, non_blocking=True)
                dh = None
                if heights_nm is not None:
                    dh = (heights_nm[b0:b1] if per_point_h else heights_nm).to(self.device, non_blocking=True)
                o = sol.solve(dw, dk, dn, dh, pol=pol, stream=st, variant=variant)
                for k in self.keys:
                    out[k][b0:b1].copy_(o[k], non_blocking=True)
        for st in self.streams:
            cur.wait_stream(st)
        return out


# ---------------------------------------------------------------- uneven batches
_POINT_DTYPE = np.dtype([
    ('n_layers', np.int32), ('n_pw', np.int32), ('world_1d', np.int32), ('pol', np.int32),
    ('order_off', np.int64), ('n_off', np.int64), ('h_off', np.int64), ('inc_off', np.int64),
    ('rt_off', np.int64), ('list_off', np.int64), ('np_off', np.int64), ('ws_off', np.int64),
    ('period', np.float64), ('period_y', np.float64), ('wl_nm', np.float64),
    ('kx', np.float64), ('ky', np.float64),
])
assert _POINT_DTYPE.itemsize == C.sizeof(_lib.EmuFilmPoint)


class FilmPoint(object):
    """One spectral point of an all-film stack, any shape.

    The arguments are what the reference's Stack(layers).calc_scat(pol)
    reads from its ThinFilm layers and Light: refractive indices bottom to
    top with each layer's ``loss`` flag already applied, finite-layer
    heights, wavelength, k_parallel (nm^-1), period(s), ``max_order_PWs``,
    the polarisation ('TE', 'TM', 'un', 'R Circ', 'L Circ') or a full
    incoming amplitude vector of length 2 Npw (sorted order).
    """

    __slots__ = ('n', 'heights', 'wl_nm', 'k_pll', 'period', 'period_y', 'max_order', 'pol',
                 'world_1d', 'incoming', '_rec')

    def __init__(self, n, heights, wl_nm, k_pll, period, max_order, pol='TE', period_y=None,
                 world_1d=False, incoming=None):
        self.n = np.asarray(n, np.complex128).reshape(-1)
        self.heights = np.asarray(heights, np.float64).reshape(-1)
        if len(self.n) < 2:
            raise ValueError('a stack needs at least a substrate and a superstrate')
        if self.heights.shape != (len(self.n) - 2,):
            raise ValueError('need one height per finite layer')
        self.wl_nm = float(wl_nm)
        self.k_pll = np.asarray(k_pll, np.float64).reshape(2)
        self.period = float(period)
        self.period_y = float(period if period_y is None else period_y)
        self.max_order = int(max_order)
        self.world_1d = bool(world_1d)
        self.incoming = None if incoming is None else np.asarray(incoming, np.complex128).reshape(-1)
        if self.incoming is None and pol not in _lib.POL:
            raise NotImplementedError('Must select from the currently implemented polarisations; '
                                      'TE, TM, R Circ, L Circ.')
        self.pol = pol
        # packing record: order-set key, then the descriptor scalars
        self._rec = ((self.max_order, self.period, self.period_y, self.world_1d), len(self.n),
                     int(self.world_1d), _lib.POL_INCOMING if self.incoming is not None else _lib.POL[pol],
                     self.period, self.period_y, self.wl_nm, float(self.k_pll[0]), float(self.k_pll[1]))


class _Grow(object):
    """A growable buffer (pinned host or device) handing out views."""

    def __init__(self, dtype, device=None, pinned=False):
        self.dtype, self.device, self.pinned = dtype, device, pinned
        self.t = None

    def get(self, n):
        n = max(int(n), 1)
        if self.t is None or self.t.numel() < n:
            cap = max(n, 2 * (self.t.numel() if self.t is not None else 0))
            if self.pinned:
                self.t = torch.empty(cap, dtype=self.dtype).pin_memory()
            else:
                self.t = torch.empty(cap, dtype=self.dtype, device=self.device)
        return self.t[:n]


class FilmVarPlan(object):
    """Host side of one uneven batch: descriptors and packed inputs in the
    solver's pinned staging buffers (valid until the solver plans again)."""

    __slots__ = ('B', 'desc', 'max_layers', 'max_pw', 'rt_len', 'list_len', 'np_len', 'ws_bytes',
                 'n_len', 'h_len', 'inc_len', 'h_desc', 'h_order', 'h_n', 'h_h', 'h_inc')


class FilmVarSolver(object):
    """All-film points of mixed shapes in one launch (``emu_film_var_batch``).

    ``plan(points)`` packs the points into pinned host staging buffers,
    ``solve(plan)`` copies them to the device, launches once and returns the
    packed device outputs, ``fetch(plan, out)`` copies those back into pinned
    host buffers, ``unpack(plan, host)`` splits host arrays per point.
    Order sets are built once per (max_order, period, period_y, world_1d)
    and shared by every point that uses them.  Staging, device and
    workspace buffers grow and are reused: one solver serves one stream.
    """

    def __init__(self, device='cuda'):
        self.device = torch.device(device)
        self._orders = {}
        self._px, self._py = [], []
        self._n_orders = 0
        self._d_orders = None
        self._ws = _Grow(torch.uint8, self.device)
        self._hs = {k: _Grow(dt, pinned=True) for k, dt in (
            ('desc', torch.uint8), ('order', torch.int32), ('n', torch.complex128),
            ('h', torch.float64), ('inc', torch.complex128))}
        self._ds = {k: _Grow(g.dtype, self.device) for k, g in self._hs.items()}
        self._out = {k: _Grow(dt, self.device) for k, dt in self._OUT}
        self._hout = {k: _Grow(dt, pinned=True) for k, dt in self._OUT}

    _OUT = (('R_net', torch.complex128), ('T_net', torch.complex128), ('a_list', torch.float64),
            ('t_list', torch.float64), ('r_list', torch.float64), ('flags', torch.int32),
            ('specular', torch.int32), ('num_prop', torch.int32))

    def _order_off(self, key):
        hit = self._orders.get(key)
        if hit is None:
            px, py = grating_orders(key[0], key[1], key[2], key[3])
            hit = (self._n_orders, len(px))
            self._orders[key] = hit
            self._px.append(px)
            self._py.append(py)
            self._n_orders += len(px)
            self._d_orders = None
        return hit

    def _device_orders(self):
        if self._d_orders is None:
            px = np.concatenate(self._px).astype(np.int32)
            py = np.concatenate(self._py).astype(np.int32)
            self._d_orders = (torch.from_numpy(px).to(self.device),
                              torch.from_numpy(py).to(self.device))
        return self._d_orders

    _REC = np.dtype([('n_layers', np.int64), ('world_1d', np.int32), ('pol', np.int32),
                     ('period', np.float64), ('period_y', np.float64), ('wl_nm', np.float64),
                     ('kx', np.float64), ('ky', np.float64)])

    def plan(self, points):
        B = len(points)
        orders = self._orders
        recs = [p._rec for p in points]
        oo = [orders.get(r[0]) or self._order_off(r[0]) for r in recs]
        sc = np.array([r[1:] for r in recs], self._REC) if B else np.zeros(0, self._REC)
        Ls = sc['n_layers']
        npw = np.fromiter((o[1] for o in oo), np.int64, B)
        desc = np.zeros(B, _POINT_DTYPE)
        for f in ('n_layers', 'world_1d', 'pol', 'period', 'period_y', 'wl_nm', 'kx', 'ky'):
            desc[f] = sc[f]
        desc['n_pw'] = npw
        desc['order_off'] = np.fromiter((o[0] for o in oo), np.int64, B)
        desc['n_off'] = np.cumsum(Ls) - Ls
        desc['h_off'] = np.cumsum(Ls - 2) - (Ls - 2)
        inc_parts, inc_off = [], 0
        if B and (sc['pol'] == _lib.POL_INCOMING).any():
            inc_offs = np.zeros(B, np.int64)
            for i in np.nonzero(sc['pol'] == _lib.POL_INCOMING)[0]:
                p = points[i]
                if p.incoming.shape != (2 * npw[i],):
                    raise ValueError('incoming must have 2 Npw = %d entries' % (2 * npw[i]))
                inc_offs[i] = inc_off
                inc_parts.append(p.incoming)
                inc_off += 2 * int(npw[i])
            desc['inc_off'] = inc_offs
        pl = FilmVarPlan()
        pl.B = B
        h_order = self._hs['order'].get(B)
        rt_len, list_len, np_len = C.c_int64(), C.c_int64(), C.c_int64()
        ws_bytes, max_l, max_pw = C.c_size_t(), C.c_int(), C.c_int()
        check(lib().emu_film_var_plan(desc.ctypes.data_as(C.c_void_p), B,
                                      C.c_void_p(h_order.data_ptr()), C.byref(rt_len),
                                      C.byref(list_len), C.byref(np_len), C.byref(ws_bytes),
                                      C.byref(max_l), C.byref(max_pw)), 'emu_film_var_plan')
        pl.desc = desc
        pl.max_layers, pl.max_pw = max_l.value, max_pw.value
        pl.rt_len, pl.list_len, pl.np_len = rt_len.value, list_len.value, np_len.value
        pl.ws_bytes = ws_bytes.value
        pl.h_order = h_order
        pl.h_desc = self._hs['desc'].get(desc.nbytes)
        pl.h_desc.numpy()[:] = desc.view(np.uint8)
        pl.n_len = int(Ls.sum())
        pl.h_n = self._hs['n'].get(pl.n_len)
        pl.h_n.numpy()[:pl.n_len] = np.concatenate([p.n for p in points]) if B else []
        pl.h_len = int((Ls - 2).sum())
        pl.h_h = self._hs['h'].get(pl.h_len)
        if pl.h_len:
            pl.h_h.numpy()[:pl.h_len] = np.concatenate([p.heights for p in points])
        pl.inc_len = inc_off
        pl.h_inc = self._hs['inc'].get(inc_off)
        if inc_off:
            pl.h_inc.numpy()[:inc_off] = np.concatenate(inc_parts)
        return pl

    def solve(self, pl, stream=None, want_num_prop=False, warps=None, variant=0):
        """Copy a plan to the device and solve it in one launch; returns
        device tensors R_net/T_net [rt_len], a_list/t_list [list_len],
        r_list/flags/specular [B] (and num_prop [np_len]), views of buffers
        this solver reuses.  warps: points (warps) per CTA, 1-8, and variant:
        register budget (EmuFilmVarBatch.variant); warps=None takes the
        autotuner's choice of both for batches of 1024 points or more, else
        8 warps, variant 0.  Results do not depend on them."""
        dev = self.device
        px, py = self._device_orders()
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        B = pl.B
        with torch.cuda.stream(s):
            d = {}
            for k, h in (('desc', pl.h_desc), ('order', pl.h_order), ('n', pl.h_n), ('h', pl.h_h),
                         ('inc', pl.h_inc)):
                d[k] = self._ds[k].get(h.numel())
                d[k].copy_(h, non_blocking=True)
            lens = dict(R_net=pl.rt_len, T_net=pl.rt_len, a_list=pl.list_len, t_list=pl.list_len,
                        r_list=B, flags=B, specular=B, num_prop=pl.np_len)
            out = {k: self._out[k].get(lens[k]) for k, _ in self._OUT
                   if k != 'num_prop' or want_num_prop}
            ws = self._ws.get(pl.ws_bytes)
            e = _lib.EmuFilmVarBatch()
            e.n_points = B
            e.max_layers, e.max_pw = pl.max_layers, pl.max_pw
            e.d_points, e.d_order = ptr(d['desc']), ptr(d['order'])
            e.d_px, e.d_py = ptr(px), ptr(py)
            e.d_n, e.d_heights_nm, e.d_incoming = ptr(d['n']), ptr(d['h']), ptr(d['inc'])
            e.d_R_net, e.d_T_net = ptr(out['R_net']), ptr(out['T_net'])
            e.d_a_list, e.d_t_list = ptr(out['a_list']), ptr(out['t_list'])
            e.d_r_list, e.d_flags = ptr(out['r_list']), ptr(out['flags'])
            e.d_specular = ptr(out['specular'])
            e.d_num_prop = ptr(out.get('num_prop'))
            e.order_len = self._n_orders
            e.n_len, e.h_len, e.inc_len = pl.n_len, pl.h_len, pl.inc_len
            e.rt_len, e.list_len, e.np_len = pl.rt_len, pl.list_len, pl.np_len

            def run(c):
                e.warps_per_cta, e.variant = int(c[0]), int(c[1])
                check(lib().emu_film_var_batch(C.byref(e), ptr(ws), C.c_size_t(ws.numel()),
                                               stream_ptr(s)), 'emu_film_var_batch')

            choice = (warps or 0, variant)
            if warps is None and B >= 1024:
                from .autotune import default_tuner, size_bucket
                shape = dict(B=size_bucket(B), max_pw=size_bucket(pl.max_pw), max_L=pl.max_layers)
                cands = [(w, v) for v in (0, 1) for w in (2, 4, 8)]
                choice = default_tuner().choose('film_var2', shape, cands, run, (0, 0), stream=s)
            run(choice)
        return out

    def fetch(self, out, stream=None):
        """Asynchronous copies of packed device outputs into pinned host
        buffers of this solver; returns numpy views (valid once the stream
        reaches this point, until the next fetch)."""
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        host = {}
        with torch.cuda.stream(s):
            for k, t in out.items():
                h = self._hout[k].get(t.numel())
                h.copy_(t, non_blocking=True)
                host[k] = h.numpy()
        return host

    @staticmethod
    def unpack(pl, host):
        """Split host copies (numpy) of the packed outputs per point."""
        res = []
        for i, d in enumerate(pl.desc):
            P, L = 2 * int(d['n_pw']), int(d['n_layers'])
            ro, lo = int(d['rt_off']), int(d['list_off'])
            r = {
                'R_net': host['R_net'][ro:ro + P], 'T_net': host['T_net'][ro:ro + P],
                'a_list': host['a_list'][lo:lo + L - 1], 't_list': host['t_list'][lo:lo + L - 1],
                'r_list': host['r_list'][i], 'flags': int(host['flags'][i]),
                'specular': int(host['specular'][i]),
            }
            if 'num_prop' in host:
                no = int(d['np_off'])
                r['num_prop'] = host['num_prop'][no:no + L + 1]
            res.append(r)
        return res
