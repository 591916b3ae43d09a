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
            # the reference's expression and order of operations (materials.py:142;
            # its sign check there tests the lambda, not the value, so never flips)
            return np.sqrt(eps_inf - wp ** 2 / (((2 * np.pi * c) / (wl_nm * 1e-9)) ** 2
                                                + 1j * wg * (2 * np.pi * c) / (wl_nm * 1e-9)))
        wl = np.asarray(wl_nm, dtype=float)
        if np.any(wl < self.data_wls[0]) or np.any(wl > self.data_wls[-1]):
            raise ValueError('wavelength outside the tabulated range')
        ns = np.asarray(self.data_ns)
        if not np.iscomplexobj(ns):
            return np.interp(wl, self.data_wls, ns)
        # interp1d's evaluation of complex data (scipy 1.18): the interval of
        # searchsorted(side='left') clipped to [1, K-1], weights of both ends
        xs = np.asarray(self.data_wls, float)
        hi = np.clip(np.searchsorted(xs, wl), 1, len(xs) - 1)
        lo = hi - 1
        x_lo, x_hi = xs[lo], xs[hi]
        return ((wl - x_lo) / (x_hi - x_lo)) * ns[hi] + ((x_hi - wl) / (x_hi - x_lo)) * ns[lo]


Air = Material(1.00 + 0.0j)


def n_batch(materials, wl_nm, losses=None):
    """Refractive indices of the layers of a stack at a batch of wavelengths,
    on the device (emu_material_n_batch): complex128 [B, L] for
    ``materials`` (L Material objects, bottom to top) at ``wl_nm`` (a CUDA
    float64 tensor [B]), each layer's imaginary part dropped where its
    ``losses`` flag is False (ThinFilm(loss=False)).  The result is the ``n``
    argument of films.FilmStackSolver.solve.  Raises ValueError for
    wavelengths outside a table, as the reference's interpolation does."""
    import ctypes as C
    import torch
    from . import _lib
    if not (torch.is_tensor(wl_nm) and wl_nm.is_cuda and wl_nm.dtype == torch.float64
            and wl_nm.dim() == 1 and wl_nm.is_contiguous()):
        raise TypeError('wl_nm must be a contiguous CUDA float64 tensor [B]')
    L = len(materials)
    losses = [True] * L if losses is None else list(losses)
    dev = wl_nm.device
    arr = (_lib.EmuMaterial * L)()
    keep = []
    for l, (m, loss) in enumerate(zip(materials, losses)):
        e = arr[l]
        e.loss = int(bool(loss))
        if m.data_wls is None:
            e.kind = _lib.MAT_CONSTANT
            v = complex(np.asarray(m.data_ns).item())
            e.n_const = _lib.EmuC128(v.real, v.imag)
        elif isinstance(m.data_wls, str):
            e.kind = _lib.MAT_DRUDE
            for i in range(3):
                e.drude[i] = float(m.data_ns[i])
        else:
            cache = getattr(m, '_device_table', None)
            if cache is None or cache[0].device != dev:
                cache = (torch.tensor(np.asarray(m.data_wls, np.float64), device=dev),
                         torch.tensor(np.asarray(m.data_ns, np.complex128), device=dev))
                m._device_table = cache
            # scipy's interp1d takes real data through numpy.interp and complex
            # data through its own weighted form; the kernel does the same
            e.kind = _lib.MAT_TABLE if np.iscomplexobj(m.data_ns) else _lib.MAT_TABLE_REAL
            e.n_rows = int(cache[0].numel())
            e.d_wl, e.d_n = _lib.ptr(cache[0]), _lib.ptr(cache[1])
            keep.append(cache)
    B = int(wl_nm.shape[0])
    out = torch.empty((B, L), dtype=torch.complex128, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.check(_lib.lib().emu_material_n_batch(arr, L, B, _lib.ptr(wl_nm), _lib.ptr(out), _lib.ptr(err),
                                               _lib.stream_ptr()), 'emu_material_n_batch')
    if int(err.item()) != 0:
        raise ValueError('wavelength outside the tabulated range')
    return out
