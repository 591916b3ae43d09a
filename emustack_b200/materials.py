"""Refractive indices of layer materials (host side).

Mirrors ``Material`` of backend/materials.py:31-186: a constant index, a
table of (wavelength_nm, n) or (wavelength_nm, n, k) rows interpolated
linearly, or Drude parameters (omega_plasma, omega_gamma, eps_inf).  The
reference's tabulated data files are not shipped here; pass the table
(e.g. ``np.loadtxt(path)``) to ``Material``.
"""
from __future__ import annotations

import numpy as np


class Material(object):
    """Refractive index n(wl_nm) of a layer material."""

    def __init__(self, n):
        if np.shape(n) == ():
            self.data_wls = None
            self.data_ns = n
        elif np.shape(n) == (3,):
            c = 299792458
            self.data_wls = 'Drude'
            self.data_ns = [n[0], n[1], n[2], c]
        else:
            n = np.asarray(n)
            if n.ndim != 2 or n.shape[1] not in (2, 3):
                raise ValueError('tabulated data must have 2 or 3 columns')
            self.data_wls = n[:, 0].astype(float)
            self.data_ns = n[:, 1] if n.shape[1] == 2 else n[:, 1] + 1j * n[:, 2]

    def n(self, wl_nm):
        """Return n at the wavelength (nm)."""
        if self.data_wls is None:
            return self.data_ns
        if isinstance(self.data_wls, str):
            wp, wg, eps_inf, c = self.data_ns
            w = (2 * np.pi * c) / (wl_nm * 1e-9)
            val = np.sqrt(eps_inf - wp ** 2 / (w ** 2 + 1j * wg * w))
            if np.imag(val) < 0:
                val = -val
            return val
        wl = np.asarray(wl_nm, dtype=float)
        if np.any(wl < self.data_wls[0]) or np.any(wl > self.data_wls[-1]):
            raise ValueError('wavelength outside the tabulated range')
        ns = np.asarray(self.data_ns)
        if np.iscomplexobj(ns):
            return np.interp(wl, self.data_wls, ns.real) + 1j * np.interp(wl, self.data_wls, ns.imag)
        return np.interp(wl, self.data_wls, ns)


Air = Material(1.00 + 0.0j)
