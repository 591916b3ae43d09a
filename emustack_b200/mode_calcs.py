"""Layer modes (mirror of backend/mode_calcs.py): ``Anallo`` for films,
``Simmo`` for nanostructured layers, and the interface memo ``r_t_mat``.

All numerics run on the GPU through libemustack_gsm.so; this module keeps
the reference's objects and attribute names so that code written against
the reference reads the same values here.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import EmuAnalloModes, check, lib, ptr, stream_ptr

pi = np.pi

# Interface memo keyed by (id(lay1), id(lay2)), as backend/mode_calcs.py:32.
# Values hold device tensors (R12, T12, R21, T21) plus host np.matrix copies
# made on first access.
_interfaces_i_have_known = {}


def _device():
    if not torch.cuda.is_available():
        raise RuntimeError('emustack_b200 needs a CUDA device (no CPU fallback)')
    return torch.device('cuda', torch.cuda.current_device())


def is_film(lay):
    """True for a homogeneous-film layer (an ``Anallo``), judged by the
    interface the GSM stage reads rather than by class: a film has analytic
    impedances (``Z``) and a specular incidence vector, a nanostructured
    layer (``Simmo``) has overlap matrices ``J`` / ``J_dag`` instead.  So the
    reference's own ``Anallo`` / ``Simmo`` objects, or any object exposing
    the same attributes, dispatch the same way as this package's."""
    return (callable(getattr(lay, 'Z', None)) and callable(getattr(lay, 'specular_incidence', None))
            and getattr(lay, 'J', None) is None)


def film_n(lay):
    """Refractive index of a film layer with its loss flag applied (the
    reference's ``Anallo.n()``, real when ``loss`` is False), as a complex."""
    return complex(np.asarray(lay.n()).item())


class Modes(object):
    """Common functionality of Simmo and Anallo (backend/mode_calcs.py:36-95)."""

    def k_pll_norm(self):
        return self.light.k_pll * self.structure.period

    def wl_norm(self):
        wl = self.light.wl_nm / self.structure.period
        if self.light.wl_nm % self.structure.period == 0:
            wl += 1e-10
        return wl

    def air_ref(self):
        return self.light._air_ref(self.structure.period, self.structure.period_y,
                                   self.structure.world_1d)

    def calc_1d_grating_orders(self, max_order):
        from .films import grating_orders
        return grating_orders(max_order, self.structure.period, self.structure.period_y, True)[0]

    def calc_2d_grating_orders(self, max_order):
        from .films import grating_orders
        return grating_orders(max_order, self.structure.period, self.structure.period_y, False)

    def prop_fwd(self, height_norm):
        """Diagonal matrix exp(i k_z h) (backend/mode_calcs.py:76-78)."""
        return np.asmatrix(np.diag(np.exp(1j * np.asarray(self.k_z) * height_norm)))

    def shear_transform(self, coords):
        """Diagonal shear matrix (backend/mode_calcs.py:80-87)."""
        alphas = np.append(self.air_ref().alphas, self.air_ref().alphas)
        if np.shape(coords) == (1,):
            return np.asmatrix(np.diag(np.exp(1j * (alphas * coords[0]))))
        betas = np.append(self.air_ref().betas, self.air_ref().betas)
        return np.asmatrix(np.diag(np.exp(1j * (alphas * coords[0] + betas * coords[1]))))

    def __del__(self):
        if _interfaces_i_have_known is not None:
            for key in list(_interfaces_i_have_known.keys()):
                if id(self) in key:
                    _interfaces_i_have_known.pop(key, None)


class Anallo(Modes):
    """Analytic plane-wave modes of a homogeneous film (backend/mode_calcs.py:99-250)."""

    def __init__(self, thin_film, light):
        self.structure = thin_film
        self.light = light
        self.max_order_PWs = light.max_order_PWs
        self.is_air_ref = False

    def calc_modes(self):
        kzs = self.calc_kz()
        self.k_z = np.append(kzs, kzs)
        self.structure.num_pw_per_pol = len(kzs)

    def n(self):
        if self.structure.loss:
            return self.structure.material.n(self.light.wl_nm)
        return self.structure.material.n(self.light.wl_nm).real

    def n_complex(self):
        """Index with the loss flag applied, as a Python complex."""
        return film_n(self)

    def k(self):
        return np.complex128(2 * pi * self.n() / self.wl_norm())

    def calc_kz(self):
        """k_z of every order, sorted by the air reference (on the GPU)."""
        from .films import grating_orders
        st = self.structure
        px, py = grating_orders(self.max_order_PWs, st.period, st.period_y, bool(st.world_1d))
        if st.world_1d not in (True, False):
            raise ValueError("must specify world_1d status of ThinFilm.")
        dev = _device()
        npw = len(px)
        d_px = torch.from_numpy(px).to(dev)
        d_py = torch.from_numpy(py).to(dev)
        wl = torch.tensor([self.light.wl_nm], dtype=torch.float64, device=dev)
        kp = torch.tensor(np.asarray(self.light.k_pll, dtype=np.float64).reshape(1, 2), device=dev)
        n = torch.tensor([self.n_complex()], dtype=torch.complex128, device=dev)
        kz = torch.empty(npw, dtype=torch.complex128, device=dev)
        alphas = torch.empty(npw, dtype=torch.float64, device=dev)
        betas = torch.empty(npw, dtype=torch.float64, device=dev)
        sort_out = torch.empty(npw, dtype=torch.int32, device=dev)
        misc = torch.empty(3, dtype=torch.int32, device=dev)
        sort_in = None
        if not self.is_air_ref:
            s = self.air_ref().sort_order
            sort_in = torch.from_numpy(np.ascontiguousarray(s, dtype=np.int32)).to(dev)
        d = EmuAnalloModes()
        d.n_points = 1
        d.n_pw = npw
        d.world_1d = int(bool(st.world_1d))
        d.period = st.period
        d.period_y = st.period_y
        d.d_px, d.d_py = ptr(d_px), ptr(d_py)
        d.d_wl_nm, d.d_k_pll, d.d_n = ptr(wl), ptr(kp), ptr(n)
        d.d_sort_in = ptr(sort_in)
        d.d_kz, d.d_alphas, d.d_betas, d.d_sort_out = ptr(kz), ptr(alphas), ptr(betas), ptr(sort_out)
        d.d_specular = C.c_void_p(misc.data_ptr())
        d.d_num_prop = C.c_void_p(misc.data_ptr() + 4)
        d.d_wood = C.c_void_p(misc.data_ptr() + 8)
        check(lib().emu_anallo_modes(C.byref(d), stream_ptr()), 'emu_anallo_modes')
        m = misc.cpu().numpy()
        self.specular_order = int(m[0])
        self.num_prop_pw_per_pol = int(m[1])
        self.wood_anomaly = bool(m[2])
        if self.wood_anomaly:
            print("Warning: selected [k_x, k_y] hits a Wood Anomaly!\n"
                  " EMUstack changed [k_x, k_y] -> (1-1e-9)*[k_x, k_y].")
        self.alphas = alphas.cpu().numpy()
        self.betas = betas.cpu().numpy() if not st.world_1d else float(betas[0].item())
        if self.is_air_ref:
            self.sort_order = sort_out.cpu().numpy().astype(np.int64)
        else:
            self.sort_order = self.air_ref().sort_order
        self._px, self._py = px, py
        return kz.cpu().numpy()

    def Z(self):
        """Wave impedances, TE half then TM half (backend/mode_calcs.py:199-218)."""
        Zcr = 1. / self.n()
        num_pw2 = int(len(self.k_z) / 2)
        k_z = self.k_z[:num_pw2]
        k_on_kz = self.k() / k_z
        return np.concatenate((Zcr * k_on_kz, Zcr / k_on_kz))

    def specular_incidence(self, pol='TE'):
        """Unit amplitude in the zeroth order (backend/mode_calcs.py:220-250)."""
        spec_TE = self.specular_order
        spec_TM = self.specular_order + self.structure.num_pw_per_pol
        tot = self.structure.num_pw_per_pol * 2
        inc = np.asmatrix(np.zeros(tot, dtype='complex128')).T
        if pol == 'TE':
            inc[spec_TE] = 1
        elif pol == 'TM':
            inc[spec_TM] = 1
        elif pol == 'un':
            inc[spec_TE] = 1 / np.sqrt(2.)
            inc[spec_TM] = 1 / np.sqrt(2.)
        elif pol == 'R Circ':
            inc[spec_TE] = 1 / np.sqrt(2.)
            inc[spec_TM] = +1j / np.sqrt(2.)
        elif pol == 'L Circ':
            inc[spec_TE] = 1 / np.sqrt(2.)
            inc[spec_TM] = -1j / np.sqrt(2.)
        else:
            raise NotImplementedError("Must select from the currently implemented polarisations; "
                                      "TE, TM, R Circ, L Circ.")
        return inc


class Simmo(Modes):
    """Bloch modes of a nanostructured layer (backend/mode_calcs.py:255-413).

    ``calc_modes`` runs the FEM eigen-solve on the GPU (2D_array layers with
    a .mail mesh); ``attach_modes`` takes modes computed elsewhere.
    """

    def __init__(self, structure, light):
        self.structure = structure
        self.light = light
        self.max_order_PWs = light.max_order_PWs
        self.prop_consts = None
        self.mode_pol = None

    def calc_modes(self, num_BMs=None, fem_block=4):
        """Bloch modes of the layer by the FEM solve on the GPU
        (emustack_b200.fem), then J and J_dag, as Simmo.calc_modes does with
        its Fortran solver (backend/mode_calcs.py:268-386): indices of the
        mesh's materials (background, inclusion_a, ...; real when loss is
        False), num_BMs = 2 Npw + 20 by default, the shift 1.1 max(Re n)^2 k0^2
        - |k_parallel|^2, prime and adjoint modes.  Needs the structure's
        ``mesh``: for 2D_array layers one that carries its boundary node types
        (Mesh.from_mail), for 1D_array layers a Mesh1D (calc_modes_1d,
        backend/mode_calcs.py:323-355)."""
        from .fem import FemMesh, FemMesh1D, FemModeSolver
        st = self.structure
        one_d = getattr(st, 'periodicity', '2D_array') == '1D_array'
        mesh = getattr(st, 'mesh', None)
        if mesh is None:
            raise ValueError('the FEM solve needs the structure\'s mesh')
        fm = getattr(st, '_fem_mesh', None)
        if fm is None or fm.mesh_id != id(mesh):
            fm = FemMesh1D.from_mesh(mesh) if one_d else FemMesh.from_mesh(mesh)
            fm.mesh_id = id(mesh)
            st._fem_mesh = fm
        wl = self.light.wl_nm
        n_types = int(np.max(mesh.type_el))
        names = ('background', 'inclusion_a', 'inclusion_b', 'inclusion_c', 'inclusion_d', 'inclusion_e')
        mats = [getattr(st, k, None) for k in names[:n_types]]
        if any(m is None for m in mats):
            raise ValueError('the mesh has %d material types; the structure defines fewer' % n_types)
        n_effs = np.array([np.asarray(m.n(wl)).item() for m in mats], dtype=np.complex128)
        if st.loss is False:
            n_effs = n_effs.real.astype(np.complex128)
        self.n_effs = n_effs
        if one_d:
            num_pw_per_pol = self.calc_1d_grating_orders(self.max_order_PWs).size
        else:
            pxs, pys = self.calc_2d_grating_orders(self.max_order_PWs)
            num_pw_per_pol = pxs.size
        nbm = num_pw_per_pol * 2 + 20 if num_BMs is None else int(num_BMs)
        if nbm <= num_pw_per_pol * 2:
            raise ValueError('You must include at least as many BMs as PWs. \nCurrently you have %i BMs < '
                             '%i PWs.' % (nbm, num_pw_per_pol * 2))
        k0 = 2 * np.pi * self.air_ref().n() / self.wl_norm()
        kp = self.k_pll_norm()
        shift = 1.1 * np.real(n_effs).max() ** 2 * k0 ** 2 - kp[0] ** 2 - kp[1] ** 2
        solver = FemModeSolver(fm, block=fem_block)
        b1, s1, b2, s2 = solver.solve_pair(n_effs, self.wl_norm(), kp, nbm, shift=float(np.real(shift)))
        self.fem_stats = solver.stats
        self.attach_modes(num_BMs=nbm, k_z=b1,
                          fields={'sol1': s1, 'sol2': s2, 'beta1': b1, 'mesh': mesh,
                                  'pp': np.ones(n_types, np.complex128)})
        return self

    def attach_modes(self, num_BMs=None, k_z=None, J=None, J_dag=None, fields=None):
        if k_z is None:
            raise ValueError('Simmo needs the Bloch-mode propagation constants k_z '
                             '(or calc_modes, which solves for them)')
        self.k_z = np.asarray(k_z, dtype=np.complex128)
        self.num_BMs = len(self.k_z) if num_BMs is None else num_BMs
        if J is not None:
            self.J = np.asmatrix(np.asarray(J, dtype=np.complex128))
            self.J_dag = np.asmatrix(np.asarray(J_dag, dtype=np.complex128))
        elif fields is not None:
            self.sol1 = fields['sol1']        # prime-mode fields, for field reconstruction
            if getattr(self.structure, 'periodicity', '2D_array') == '1D_array':
                from .overlap import overlap_from_fields_1d
                self.J, self.J_dag = overlap_from_fields_1d(self, fields)
            else:
                from .overlap import overlap_from_fields
                self.J, self.J_dag = overlap_from_fields(self, fields)
        else:
            raise ValueError('Simmo needs J / J_dag or mode fields')
