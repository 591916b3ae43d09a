"""The whole per-wavelength GSM of a stack with one nanostructured layer, for a
batch of wavelengths, as one chain of device calls that can be recorded in a
CUDA graph.

Stack (bottom to top): film substrate n_sub / one periodic nanostructured
layer (P2 mode fields of `nval` Bloch modes on a mesh, height h) / film
superstrate n_sup.  Per wavelength the chain is the reference's
  Anallo.calc_kz for the air reference and the substrate
                                           (backend/mode_calcs.py:116-186)
  orthogonal.f + normalisation.f           (adjoint-mode normalisation)
  J_overlap.f, J_dagger_overlap.f          (backend/mode_calcs.py:371-386)
  r_t_mat_anallo, r_t_mat_tf_ns            (backend/mode_calcs.py:451-515)
  Stack.calc_scat cascade + fluxes         (backend/stack.py:162-426)
run here for all wavelengths of the batch at once: ~13 library launches per
wavelength of the overlap stage plus a few batched launches for the rest.
``capture()`` records the chain once into a CUDA graph over static input
and output buffers; ``replay()`` then re-runs it with one graph launch after
``load()`` has copied new inputs in.  Mode fields come from the caller (the
FEM eigen-solve stays outside the GSM stage).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import EmuAnalloModes, check, lib, ptr, stream_ptr
from .dense import DenseLayer, DenseStackSolver, film_interface, interface_dense
from .films import grating_orders
from .overlap import DeviceMesh, mode_normalisation, overlap_batch

c128 = torch.complex128


class NanoStackPipeline(object):
    def __init__(self, mesh, period, max_order, nval, batch, height_nm, n_sub=1.46, n_sup=1.0,
                 pol='TE', precision='fp64', pp=None, device='cuda'):
        self.dev = torch.device(device)
        self.period = float(period)
        self.B, self.M = int(batch), int(nval)
        self.max_order = int(max_order)
        self.dm = DeviceMesh(mesh, self.dev)
        px, py = grating_orders(self.max_order, self.period, self.period)
        self.px_h, self.py_h = px, py
        self.npw = len(px)
        self.P = 2 * self.npw
        self.d_px = torch.from_numpy(px).to(self.dev)
        self.d_py = torch.from_numpy(py).to(self.dev)
        self.hn = float(height_nm) / self.period
        self.n_sub, self.n_sup = complex(n_sub), complex(n_sup)
        self.pol, self.precision = pol, precision
        n_types = int(np.max(mesh.type_el))
        pp = np.ones(n_types, np.complex128) if pp is None else np.asarray(pp, np.complex128)
        self.pp = torch.from_numpy(pp).to(self.dev)
        B, M, nel = self.B, self.M, self.dm.nel
        z = lambda *s, dt=torch.float64: torch.zeros(s, dtype=dt, device=self.dev)
        # static inputs
        self.wl = z(B)
        self.k_pll = z(B, 2)
        self.sol1 = z(B, nel, M, 13, 3, dt=c128)
        self.sol2 = z(B, nel, M, 13, 3, dt=c128)
        self.beta1 = z(B, M, dt=c128)
        self.graph = None
        self.out = None
        self.solver = DenseStackSolver(self.dev)

    def load(self, wl_nm, k_pll, sol1, sol2, beta1):
        """Copy one batch of inputs into the static buffers (any device)."""
        self.wl.copy_(torch.as_tensor(wl_nm, dtype=torch.float64), non_blocking=True)
        self.k_pll.copy_(torch.as_tensor(k_pll, dtype=torch.float64).reshape(self.B, 2), non_blocking=True)
        self.sol1.copy_(sol1, non_blocking=True)
        self.sol2.copy_(sol2, non_blocking=True)
        self.beta1.copy_(beta1, non_blocking=True)

    def _films(self, n, sort_in):
        B, npw = self.B, self.npw
        kz = torch.empty((B, npw), dtype=c128, device=self.dev)
        sort_out = torch.empty((B, npw), dtype=torch.int32, device=self.dev)
        spec = torch.empty(B, dtype=torch.int32, device=self.dev)
        nprop = torch.empty(B, dtype=torch.int32, device=self.dev)
        nn = torch.full((B,), n, dtype=c128, device=self.dev)
        d = EmuAnalloModes()
        d.n_points, d.n_pw, d.world_1d = B, npw, 0
        d.period = d.period_y = self.period
        d.d_px, d.d_py = ptr(self.d_px), ptr(self.d_py)
        d.d_wl_nm, d.d_k_pll, d.d_n = ptr(self.wl), ptr(self.k_pll), ptr(nn)
        d.d_sort_in = ptr(sort_in)
        d.d_kz, d.d_sort_out, d.d_specular, d.d_num_prop = ptr(kz), ptr(sort_out), ptr(spec), ptr(nprop)
        check(lib().emu_anallo_modes(C.byref(d), stream_ptr()), 'emu_anallo_modes')
        return kz, nn, sort_out, spec, nprop

    def forward(self):
        """Run the chain on the current stream (no host synchronisation);
        returns device tensors R_net [B,P,P], T_net [B,M_sub,P], a_list,
        t_list [B,2], r_list [B], fluxes, flags and the interface info."""
        B = self.B
        wln = self.wl / self.period
        k0 = 2 * np.pi / wln
        bloch = self.k_pll * self.period
        kz_air, n_air, sort_air, spec, np_air = self._films(self.n_sup, None)
        kz_sub, n_sub, _, _, np_sub = self._films(self.n_sub, sort_air)
        _, scale, _ = mode_normalisation(self.dm, self.pp, k0, self.beta1, self.sol1, self.sol2)
        J, Jd, _ = overlap_batch(self.dm, self.d_px, self.d_py, self.max_order, bloch, k0, self.sol1,
                                 self.sol2, area_norm=1.0, dy=1.0, scale2=scale,
                                 precision=self.precision, check_error=False)
        R12, T12, R21, T21, info = interface_dense(kz_air, n_air, wln, J, Jd)
        Rs, Ts = film_interface(kz_air, n_air, kz_sub, n_sub, wln)
        Ra, Ta = film_interface(kz_air, n_air, kz_air, n_air, wln)
        layers = [DenseLayer(Rs, Ts, -Rs, Ts, False),
                  DenseLayer(R12, T12, R21, T21, True, self.beta1, self.hn),
                  DenseLayer(Ra, Ta, -Ra, Ta, False)]
        nprop = torch.stack([np_air, np_air, np_sub], dim=1).contiguous()
        out = self.solver.solve(layers, self.P, pol=self.pol, specular=spec, num_prop=nprop)
        out['interface_info'] = info
        return out

    def capture(self):
        """Warm up (allocations, autotuning, constant tables) and record the
        chain in a CUDA graph."""
        s = torch.cuda.Stream(self.dev)
        s.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(s):
            self.forward()
        torch.cuda.current_stream(self.dev).wait_stream(s)
        torch.cuda.synchronize(self.dev)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.out = self.forward()
        return self.out

    def replay(self):
        self.graph.replay()
        return self.out
