"""``Stack``: net scattering matrices and energy fluxes of a multilayer
(mirror of backend/stack.py).

``Stack(layers, heights_nm, shears).calc_scat(pol, incoming_amplitudes,
calc_fluxes, save_scat_list)`` fills the same attributes as the reference:
``R_net``, ``T_net`` (np.matrix, complex128), ``a_list``, ``t_list``,
``r_list``, ``vec_coef_down``, ``vec_coef_up``, optionally ``tnet_list`` /
``rnet_list``, and ``R12, T12, R21, T21`` on every layer.  Layers are
ordered bottom (substrate) to top (superstrate).

All-film stacks run through the fused film kernel (one launch); stacks with
nanostructured layers run the dense GPU path (interfaces, cascade, fluxes).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .mode_calcs import film_n, is_film


class Stack(object):
    """A stack of layers evaluated at one frequency (backend/stack.py:26-61)."""

    def __init__(self, layers, heights_nm=None, shears=None):
        self.layers = tuple(layers)
        self._heights_nm = heights_nm
        self.shears = shears
        self.period = float(layers[0].structure.period)
        self.period_y = float(layers[0].structure.period_y)
        self._check_periods_are_consistent()
        if self._heights_nm is not None:
            for i_lay, lay in enumerate(self.layers[1:-1]):
                lay.structure.height_nm = heights_nm[i_lay]

    def heights_nm(self):
        if self._heights_nm is not None:
            return self._heights_nm
        return [float(lay.structure.height_nm) for lay in self.layers[1:-1]]

    def heights_norm(self):
        return [h / self.period for h in self.heights_nm()]

    def total_height(self):
        return sum(self.heights_nm())

    def structures(self):
        return (lay.structure for lay in self.layers)

    def _check_periods_are_consistent(self):
        for lay in self.layers:
            assert lay.structure.period == self.period, \
                "All layers in a multilayer stack must have the same period."
            assert lay.structure.period_y == self.period_y, \
                "All layers in a multilayer stack must have the same period_y."

    # ------------------------------------------------------------------
    def calc_scat(self, pol='TE', incoming_amplitudes=None, calc_fluxes=True,
                  save_scat_list=False):
        """Net R/T matrices and energy fluxes (backend/stack.py:162-426)."""
        self._check_periods_are_consistent()
        all_films = all(is_film(l) for l in self.layers)
        if all_films and not save_scat_list:
            self._calc_scat_films(pol, incoming_amplitudes, calc_fluxes)
        else:
            from .dense import calc_scat_dense
            calc_scat_dense(self, pol, incoming_amplitudes, calc_fluxes, save_scat_list)

    def _calc_scat_films(self, pol, incoming_amplitudes, calc_fluxes):
        from .films import FilmStackSolver
        lay0 = self.layers[0]
        light = lay0.light
        L = len(self.layers)
        st0 = lay0.structure
        solver = FilmStackSolver(L, light.max_order_PWs, self.period, self.period_y,
                                 bool(st0.world_1d))
        dev = solver.device
        wl = torch.tensor([light.wl_nm], dtype=torch.float64, device=dev)
        kp = torch.tensor(np.asarray(light.k_pll, np.float64).reshape(1, 2), device=dev)
        n = torch.tensor([[film_n(l) for l in self.layers]], dtype=torch.complex128, device=dev)
        hs = torch.tensor(np.asarray(self.heights_nm(), dtype=np.float64), device=dev)
        inc = None
        if incoming_amplitudes is not None:
            inc = torch.tensor(np.asarray(incoming_amplitudes, dtype=np.complex128).reshape(1, -1),
                               device=dev)
        sh = None
        if self.shears is not None:
            sh = torch.tensor(np.array([np.asarray(s, dtype=np.float64) for s in self.shears]),
                              device=dev)
        out = solver.solve(wl, kp, n, hs, pol=pol, incoming=inc, shears=sh,
                           want=('layer_rt', 'vec_coef', 'fluxes', 'num_prop'))
        o = {k: v.cpu().numpy() for k, v in out.items()}
        P = solver.P
        self.R_net = np.asmatrix(np.diag(o['R_net'][0]))
        self.T_net = np.asmatrix(np.diag(o['T_net'][0]))
        for i, lay in enumerate(self.layers):
            R12 = np.asmatrix(np.diag(o['layer_rt'][0, i, 0]))
            T12 = np.asmatrix(np.diag(o['layer_rt'][0, i, 1]))
            lay.R12, lay.T12, lay.R21, lay.T21 = R12, T12, -R12, T12
        if not calc_fluxes:
            return
        flags = int(o['flags'][0])
        self.vec_coef_down = [np.asmatrix(v.reshape(P, 1)) for v in o['vec_coef_down'][0]]
        self.vec_coef_up = [np.asmatrix(v.reshape(P, 1)) for v in o['vec_coef_up'][0]]
        if flags & _lib.PT_NO_PROP_SUB:
            print("Warning: there are no propagating modes in the semi-inf \n substrate therefore "
                  "cannot calculate energy fluxes here.")
            self.a_list = np.zeros(L - 2)
            self.r_list = np.zeros(L - 2)
            self.t_list = np.zeros(L - 2)
        else:
            self.a_list = [float(v) for v in o['a_list'][0]]
            self.t_list = [float(v) for v in o['t_list'][0]]
            self.r_list = [float(o['r_list'][0])]
        f = o['fluxes'][0]
        self.down_fluxes = [f[0, 0]] + [complex(f[i, 0], f[i, 1]) for i in range(1, L - 1)] + \
            ([f[L - 1, 0]] if not flags & _lib.PT_NO_PROP_SUB else [])
        self.up_flux = [f[L, 0]]
