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
              want=(), stream=None):
        """Solve a batch on the device.

        wl_nm   float64 [B]           k_pll float64 [B, 2] (nm^-1)
        n       complex128 [B, L]     (loss already applied)
        heights float64 [L-2] or [B, L-2] (nm)
        incoming complex128 [B, P] or None (then ``pol`` selects the
        specular incidence of backend/mode_calcs.py:220-250)
        shears  float64 [L, ncoord] or None
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
        check(L.emu_film_stack_batch(C.byref(d), ptr(ws), C.c_size_t(ws.numel()), stream_ptr(stream)),
              'emu_film_stack_batch')
        return out
