"""Layer and light objects (mirror of backend/objects.py).

``Light``, ``ThinFilm`` and ``NanoStruct`` keep the reference's constructor
arguments for everything the GSM stage reads.  Meshing (gmsh) and the FEM
mode solve are not part of this package: a ``NanoStruct`` gets its Bloch
modes from the caller, either as ready overlap matrices (k_z, J, J_dag, the
outputs of the reference's ``Simmo.calc_modes``) or as P2 mode fields on a
mesh, from which the GPU computes J and J_dag.
"""
from __future__ import annotations

import numpy as np

from . import materials
from .mode_calcs import Anallo, Simmo


class Light(object):
    """Incident light (backend/objects.py:1681-1777).

    ``wl_nm`` and ``k_parallel`` are unnormalised (nm, nm^-1).  Angles below
    1e-5 degrees are nudged to 1e-5 as in the reference.
    """

    def __init__(self, wl_nm, max_order_PWs=2, k_parallel=None, theta=None, phi=None, n_inc=1.):
        if np.imag(wl_nm) != 0:
            raise ValueError('complex wavelengths are not supported by the GPU GSM stage')
        self.wl_nm = float(np.real(wl_nm))
        self._air_anallos = {}
        self.max_order_PWs = max_order_PWs
        if theta is None and k_parallel is None:
            raise ValueError("Specify incident angle either by \n k_parallel OR by theta, phi and n_inc.")
        if theta is None:
            self.k_pll = np.array(k_parallel, dtype='float64')
            if np.abs(self.k_pll[0]) == 0 or np.abs(self.k_pll[1]) == 0:
                print("Warning: a component of k_parallel is exactly zero, \n"
                      "this can lead to degeneracies and errors.")
        else:
            if k_parallel is not None or phi is None:
                raise ValueError("Specify incident angle either by \n k_parallel OR by theta, phi and n_inc.")
            if abs(theta) < 1e-5:
                theta += 1e-5
            if abs(phi) < 1e-5:
                phi += 1e-5
            k = 2 * np.pi * np.real(n_inc) / self.wl_nm
            theta *= np.pi / 180
            phi *= np.pi / 180
            self.k_pll = k * np.sin(theta) * np.array([np.cos(phi), np.sin(phi)], dtype='float64')

    def _air_ref(self, period, period_y, world_1d):
        """Anallo of free space for this light (cached per period)."""
        if period in self._air_anallos:
            return self._air_anallos[period]
        air = ThinFilm(period=period, period_y=period_y, material=materials.Air, world_1d=world_1d)
        an = Anallo(air, self)
        an.is_air_ref = True
        an.calc_modes()
        self._air_anallos[period] = an
        return an


class ThinFilm(object):
    """Homogeneous film (backend/objects.py:1611-1669)."""

    def __init__(self, period, period_y=None, height_nm=1.0, num_pw_per_pol=0, world_1d=False,
                 material=materials.Material(3.0 + 0.001), loss=True):
        self.period = float(period)
        self.period_y = float(period if period_y is None else period_y)
        self.world_1d = world_1d
        self.height_nm = height_nm
        self.num_pw_per_pol = num_pw_per_pol
        self.material = material
        self.loss = loss

    def calc_modes(self, light):
        an = Anallo(self, light)
        an.calc_modes()
        return an


class NanoStruct(object):
    """Periodic nanostructured layer (backend/objects.py:42-364, GSM-relevant part).

    Keyword arguments the GSM stage reads: ``periodicity`` ('1D_array' or
    '2D_array'), ``period``, ``period_y``, ``height_nm``, ``world_1d``,
    ``loss`` and the materials.  ``mesh`` (an ``emustack_b200.mesh.Mesh``)
    is needed only when J and J_dag are computed from mode fields.
    """

    def __init__(self, periodicity, period, diameter1=0, period_y=None, height_nm=100.0,
                 world_1d=None, loss=True, background=materials.Material(1.0 + 0.0j),
                 inclusion_a=materials.Material(1.0 + 0.0j), mesh=None, **kwargs):
        if periodicity not in ('1D_array', '2D_array'):
            raise ValueError("Must be simulating either a '1D_array' or a '2D_array'.")
        self.periodicity = periodicity
        self.period = float(period)
        self.period_y = float(period if period_y is None else period_y)
        self.diameter1 = diameter1
        self.height_nm = height_nm
        self.loss = loss
        self.background = background
        self.inclusion_a = inclusion_a
        self.mesh = mesh
        for k, v in kwargs.items():
            setattr(self, k, v)
        if world_1d is None:
            self.world_1d = periodicity == '1D_array'
        else:
            self.world_1d = world_1d

    def calc_modes(self, light, num_BMs=None, k_z=None, J=None, J_dag=None, fields=None):
        """Bloch modes of the layer as a ``Simmo``: with no modes given, the
        FEM solve on the GPU (2D_array layers whose ``mesh`` came from a .mail
        file, Simmo.calc_modes); else the modes given are attached.

        Either ``k_z`` (M,), ``J`` (P, M) and ``J_dag`` (M, P) -- J already
        divided by the area ratio as in backend/mode_calcs.py:384-386 -- or
        ``k_z`` and ``fields`` = dict(sol1=..., sol2=...) of P2 mode fields on
        ``self.mesh``; J and J_dag are then computed on the GPU.
        """
        sim = Simmo(self, light)
        if k_z is None and J is None and fields is None:
            return sim.calc_modes(num_BMs)
        sim.attach_modes(num_BMs=num_BMs, k_z=k_z, J=J, J_dag=J_dag, fields=fields)
        return sim
