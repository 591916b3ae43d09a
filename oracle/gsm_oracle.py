"""CPU oracle for the EMUstack generalised scattering-matrix (GSM) stage.

TEST INFRASTRUCTURE ONLY.  This module is a plain-numpy restatement of the
reference's FP64 algorithm and is used as the checker: by ``tests/``, by
``__graft_entry__.smoke()`` and by the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py``.  The product package ``emustack_b200`` never imports it.

Every function follows one piece of the reference and cites it (paths are
relative to the EMUstack source tree):

* plane-wave order sets      backend/mode_calcs.py:55-74
* Anallo k_z / sort / Z      backend/mode_calcs.py:41-47, 116-250
* Light k_parallel           backend/objects.py:1703-1743
* interface S-matrices       backend/mode_calcs.py:451-515
* propagation / shear        backend/mode_calcs.py:76-87
* cascade + energy fluxes    backend/stack.py:162-426

Numerics mirror the reference: complex128 throughout, dense ``np.linalg.solve``
(LAPACK zgesv) for every solve, and the same operation order wherever the
order changes rounding (e.g. ``Zcr / (k/k_z)`` for TM impedances).

Parity of this restatement is pinned against the reference's stored golden
results (tests/ref/case_{0..5}.npz and tests/ref/case_*/*.txt) through the
fixtures under ``tests/golden/``.
"""
from __future__ import annotations

import numpy as np

PI = np.pi

POLARISATIONS = ('TE', 'TM', 'un', 'R Circ', 'L Circ')


# ---------------------------------------------------------------------------
# Light and plane-wave bookkeeping
# ---------------------------------------------------------------------------

def k_parallel_from_angles(wl_nm, theta, phi, n_inc=1.0):
    """k_parallel (nm^-1) from incidence angles (degrees).

    backend/objects.py:1729-1743: angles below 1e-5 degrees are nudged by
    +1e-5 to avoid the normal-incidence degeneracy.
    """
    if abs(theta) < 1e-5:
        theta += 1e-5
    if abs(phi) < 1e-5:
        phi += 1e-5
    k = 2 * np.pi * np.real(n_inc) / wl_nm
    theta *= np.pi / 180
    phi *= np.pi / 180
    return k * np.sin(theta) * np.array([np.cos(phi), np.sin(phi)], dtype='float64')


def wl_norm(wl_nm, period):
    """Normalised wavelength with the Wood-anomaly nudge (mode_calcs.py:41-47)."""
    wl = wl_nm / period
    if wl_nm % period == 0:
        wl += 1e-10
    return wl


def grating_orders_2d(max_order, period, period_y):
    """(px, py) orders inside the disc, in the reference's order (mode_calcs.py:61-74)."""
    pxs = pys = np.arange(-max_order, max_order + 1)
    pys_mesh, pxs_mesh = np.meshgrid(pys, pxs)
    dx = period
    dy = period_y
    low_ord = ((pxs_mesh / dx) ** 2 + (pys_mesh / dy) ** 2 <=
               (max_order / max(dx, dy)) ** 2)
    return pxs_mesh[low_ord], pys_mesh[low_ord]


def grating_orders_1d(max_order):
    """px orders of a 1D grating (mode_calcs.py:55-59)."""
    return np.arange(-max_order, max_order + 1)


class FilmModes(object):
    """Analytic plane-wave modes of a homogeneous film (reference: ``Anallo``).

    Attributes mirror the reference object: ``k_z`` (length 2*Npw, TE half then
    TM half), ``alphas``/``betas`` (unsorted), ``sort_order``,
    ``specular_order``, ``num_prop_pw_per_pol``, ``num_pw_per_pol``.
    """

    def __init__(self, n, wl_nm, k_pll, period, period_y=None, max_order=2,
                 world_1d=False, loss=True, air=None, is_air_ref=False):
        self.n_raw = complex(n)
        self.loss = loss
        self.n_val = self.n_raw if loss else self.n_raw.real
        self.wl_nm = float(wl_nm)
        self.k_pll = np.asarray(k_pll, dtype=np.float64)
        self.period = float(period)
        self.period_y = float(period if period_y is None else period_y)
        self.max_order = int(max_order)
        self.world_1d = bool(world_1d)
        self.is_air_ref = is_air_ref
        self.air = air
        kzs = self.calc_kz()
        self.num_pw_per_pol = len(kzs)
        self.k_z = np.append(kzs, kzs)

    # mode_calcs.py:38-39
    def k_pll_norm(self):
        return self.k_pll * self.period

    # mode_calcs.py:195-197
    def k(self):
        return np.complex128(2 * PI * self.n_val / wl_norm(self.wl_nm, self.period))

    # mode_calcs.py:116-186
    def calc_kz(self):
        d = 1
        dy = self.period_y / self.period
        if self.world_1d:
            pxs = grating_orders_1d(self.max_order)
            pys = None
            alpha0, beta0 = self.k_pll_norm()
            alphas = alpha0 + pxs * 2 * PI / d
            betas = beta0
        else:
            pxs, pys = grating_orders_2d(self.max_order, self.period, self.period_y)
            alpha0, beta0 = self.k_pll_norm()
            alphas = alpha0 + pxs * 2 * PI / d
            betas = beta0 + pys * 2 * PI / dy
        k_z_unsrt = np.sqrt(self.k() ** 2 - alphas ** 2 - betas ** 2)
        if np.count_nonzero(k_z_unsrt) != k_z_unsrt.shape[0]:
            # Wood anomaly: shrink k_parallel by (1 - 1e-9) (mode_calcs.py:147-162)
            self.wood_anomaly = True
            alpha0, beta0 = (1 - 1e-9) * self.k_pll_norm()
            alphas = alpha0 + pxs * 2 * PI / d
            if self.world_1d:
                betas = beta0
            else:
                betas = beta0 + pys * 2 * PI / dy
            k_z_unsrt = np.sqrt(self.k() ** 2 - alphas ** 2 - betas ** 2)
        else:
            self.wood_anomaly = False
        self.alphas = alphas
        self.betas = betas
        self.pxs = pxs
        self.pys = pys
        if self.is_air_ref:
            s = np.argsort(-1 * k_z_unsrt.real + k_z_unsrt.imag)
        else:
            s = self.air.sort_order
        self.sort_order = s
        if self.world_1d:
            self.specular_order = np.nonzero(pxs[s] == 0)[0][0]
        else:
            self.specular_order = np.nonzero((pxs[s] == 0) * (pys[s] == 0))[0][0]
        self.num_prop_pw_per_pol = int((k_z_unsrt.imag == 0).sum())
        return k_z_unsrt[s]

    # mode_calcs.py:199-218
    def Z(self):
        Zcr = 1. / self.n_val
        num_pw2 = int(len(self.k_z) / 2)
        k_z = self.k_z[:num_pw2]
        k_on_kz = self.k() / k_z
        return np.concatenate((Zcr * k_on_kz, Zcr / k_on_kz))

    # mode_calcs.py:220-250
    def specular_incidence(self, pol='TE'):
        return specular_incidence(self.specular_order, self.num_pw_per_pol, pol)

    def prop_fwd(self, height_norm):
        return prop_fwd(self.k_z, height_norm)


def make_air_ref(wl_nm, k_pll, period, period_y=None, max_order=2, world_1d=False):
    """Air reference film for one Light (objects.py:1745-1777)."""
    return FilmModes(1.0 + 0.0j, wl_nm, k_pll, period, period_y, max_order,
                     world_1d, loss=False, is_air_ref=True)


def specular_incidence(specular_order, num_pw_per_pol, pol='TE'):
    """Unit incident amplitude vector in the zeroth order (mode_calcs.py:220-250)."""
    spec_TE = specular_order
    spec_TM = specular_order + num_pw_per_pol
    inc = np.zeros((2 * num_pw_per_pol, 1), dtype='complex128')
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
        raise NotImplementedError("Must select from the currently implemented "
                                  "polarisations; TE, TM, R Circ, L Circ.")
    return inc


def prop_fwd(k_z, height_norm):
    """Diagonal propagation exp(i k_z h) as a dense matrix (mode_calcs.py:76-78)."""
    return np.diag(np.exp(1j * np.asarray(k_z) * height_norm))


def shear_transform(alphas, betas, coords):
    """Diagonal shear exp(i(alpha*sx + beta*sy)) (mode_calcs.py:80-87).

    As in the reference, ``alphas``/``betas`` are the air reference's
    UNSORTED arrays, repeated for both polarisations.
    """
    a = np.append(alphas, alphas)
    if np.shape(coords) == (1,):
        return np.diag(np.exp(1j * (a * coords[0])))
    b = np.append(betas, betas)
    return np.diag(np.exp(1j * (a * coords[0] + b * coords[1])))


# ---------------------------------------------------------------------------
# Interface scattering matrices
# ---------------------------------------------------------------------------

def r_t_mat_anallo(Z1, Z2):
    """Film/film interface (mode_calcs.py:451-477): diagonal Fresnel matrices."""
    R12 = np.diag((Z2 - Z1) / (Z2 + Z1))
    T12 = np.diag(2. * np.sqrt(Z2) * np.sqrt(Z1) / (Z2 + Z1))
    return R12, T12, -R12, T12


def r_t_mat_tf_ns(Z1, J, J_dag):
    """Film/nanostructure interface (mode_calcs.py:480-515).

    ``J`` is (P, M), ``J_dag`` is (M, P), ``Z1`` the film impedances (P,).
    Returns R12 (P,P), T12 (M,P), R21 (M,M), T21 (P,M).
    """
    J = np.asarray(J)
    J_dag = np.asarray(J_dag)
    Z1_sqrt_inv = np.sqrt(1 / np.asarray(Z1)).reshape((1, -1))
    if Z1_sqrt_inv.shape[1] != J.shape[0]:
        raise ValueError("Scattering matrices of layers are not consistent,"
                         "\nsome layers are 1D and others 2D. Check that world_1d status.")
    A = Z1_sqrt_inv.T * J
    B = J_dag * Z1_sqrt_inv
    denominator = np.eye(len(B)) + B @ A
    den_inv_times_B = np.linalg.solve(denominator, B)
    R12 = -np.eye(len(A)) + 2 * A @ den_inv_times_B
    T12 = 2 * den_inv_times_B
    R21 = np.linalg.solve(denominator, (np.eye(len(B)) - B @ A))
    T21 = 2 * A @ np.linalg.inv(denominator)
    return R12, T12, R21, T21


# ---------------------------------------------------------------------------
# Layers and the stack
# ---------------------------------------------------------------------------

class OracleLayer(object):
    """One layer of an oracle stack.

    kind 'film': analytic modes (``modes`` is a FilmModes).
    kind 'struct': a nanostructured layer given by its air-interface matrices
    (R12, T12, R21, T21) and Bloch-mode k_z, or by J / J_dag (the interface is
    then computed with ``r_t_mat_tf_ns``).
    """

    def __init__(self, kind, k_z, height_nm=None, modes=None,
                 rt=None, J=None, J_dag=None):
        self.kind = kind
        self.k_z = np.asarray(k_z)
        self.height_nm = height_nm
        self.modes = modes
        self.rt = rt
        self.J = J
        self.J_dag = J_dag

    @property
    def num_prop_pw_per_pol(self):
        return self.modes.num_prop_pw_per_pol

    def interface(self, air):
        if self.rt is not None:
            return self.rt
        if self.kind == 'film':
            if len(air.k_z) != len(self.modes.k_z):
                raise ValueError("Need the same number of plane waves")
            self.rt = r_t_mat_anallo(air.Z(), self.modes.Z())
        else:
            self.rt = r_t_mat_tf_ns(air.Z(), self.J, self.J_dag)
        return self.rt


def film_layer(n, wl_nm, k_pll, period, air, height_nm=None, period_y=None,
               max_order=2, world_1d=False, loss=True):
    m = FilmModes(n, wl_nm, k_pll, period, period_y, max_order, world_1d,
                  loss=loss, air=air)
    return OracleLayer('film', m.k_z, height_nm=height_nm, modes=m)


class StackResult(object):
    pass


def calc_scat(layers, air, period, pol='TE', incoming_amplitudes=None,
              calc_fluxes=True, shears=None, heights_nm=None):
    """Net scattering matrices and energy fluxes of a stack (stack.py:162-426).

    ``layers`` are ordered bottom (substrate) to top (superstrate), as in the
    reference.  Returns a StackResult with ``R_net``, ``T_net``, ``a_list``,
    ``t_list``, ``r_list``, ``vec_coef_down``, ``vec_coef_up``,
    ``down_fluxes``, ``up_flux`` and the per-layer interface matrices.
    """
    out = StackResult()
    nl = len(layers)
    if heights_nm is None:
        heights_nm = [float(l.height_nm) for l in layers[1:-1]]
    r12_list, r21_list, t12_list, t21_list, P_list = [], [], [], [], []
    for st1 in layers:
        R12, T12, R21, T21 = st1.interface(air)
        r12_list.append(R12)
        r21_list.append(R21)
        t12_list.append(T12)
        t21_list.append(T21)
    out.interfaces = list(zip(r12_list, t12_list, r21_list, t21_list))

    PW_pols = int(np.shape(R12)[0])
    neq_PW = int(PW_pols / 2.0)
    I_air = np.eye(PW_pols, dtype='D')

    tnet_list, rnet_list = [], []
    tnet = t12_list[0]
    rnet = r12_list[0]
    tnet_list.append(tnet)
    rnet_list.append(rnet)
    inv_t21_list, inv_t12_list = [], []

    def shear_Q(coord_diff):
        return (shear_transform(air.alphas, air.betas, coord_diff),
                shear_transform(air.alphas, air.betas, -1 * coord_diff))

    for i in range(1, nl - 1):
        lay = layers[i]
        # stack.py:229-247 -- air gap below layer i
        if shears is None:
            to_invert = I_air - r12_list[i] @ rnet
            inverted_t21 = np.linalg.solve(to_invert, t21_list[i])
            tnet = tnet @ inverted_t21
            rnet = r21_list[i] + t12_list[i] @ rnet @ inverted_t21
        else:
            coord_diff = np.asarray(shears[i - 1]) - np.asarray(shears[i])
            Q, Q_inv = shear_Q(coord_diff)
            to_invert = I_air - r12_list[i] @ Q_inv @ rnet @ Q
            inverted_t21 = np.linalg.solve(to_invert, t21_list[i])
            tnet = tnet @ Q @ inverted_t21
            rnet = r21_list[i] + t12_list[i] @ Q_inv @ rnet @ Q @ inverted_t21
        inv_t21_list.append(inverted_t21)
        tnet_list.append(tnet)
        rnet_list.append(rnet)
        # stack.py:249-262 -- through layer i
        P = prop_fwd(lay.k_z, heights_nm[i - 1] / period)
        I_TF = np.eye(len(P), dtype='D')
        to_invert = I_TF - r21_list[i] @ P @ rnet @ P
        inverted_t12 = np.linalg.solve(to_invert, t12_list[i])
        P_inverted_t12 = P @ inverted_t12
        tnet = tnet @ P_inverted_t12
        rnet = r12_list[i] + t21_list[i] @ P @ rnet @ P_inverted_t12
        P_list.append(P)
        inv_t12_list.append(inverted_t12)
        tnet_list.append(tnet)
        rnet_list.append(rnet)

    # stack.py:263-278 -- into the superstrate
    if shears is None:
        to_invert = I_air - r12_list[-1] @ rnet
        inverted_t21 = np.linalg.solve(to_invert, t21_list[-1])
        tnet = tnet @ inverted_t21
        rnet = r21_list[-1] + t12_list[-1] @ rnet @ inverted_t21
    else:
        coord_diff = np.asarray(shears[-1])
        Q, Q_inv = shear_Q(coord_diff)
        to_invert = I_air - r12_list[-1] @ Q_inv @ rnet @ Q
        inverted_t21 = np.linalg.solve(to_invert, t21_list[-1])
        tnet = tnet @ Q @ inverted_t21
        rnet = r21_list[-1] + t12_list[-1] @ Q_inv @ rnet @ Q @ inverted_t21
    inv_t21_list.append(inverted_t21)
    tnet_list.append(tnet)
    rnet_list.append(rnet)
    out.R_net, out.T_net = rnet, tnet
    out.tnet_list, out.rnet_list = tnet_list, rnet_list
    if not calc_fluxes:
        return out

    # stack.py:289-426 -- energy fluxes, top to bottom
    t_list, r_list, a_list = [], [], []
    num_prop_air = air.num_prop_pw_per_pol
    num_prop_in = layers[-1].num_prop_pw_per_pol
    down_fluxes, up_flux = [], []
    vec_coef_down, vec_coef_up = [], []
    U_mat = flux_weight_matrix(PW_pols, num_prop_air)
    if incoming_amplitudes is None:
        d_minus = layers[-1].modes.specular_incidence(pol)
    else:
        d_minus = np.asarray(incoming_amplitudes, dtype=np.complex128).reshape(-1, 1)
    flux_TE = np.linalg.norm(d_minus[0:num_prop_in]) ** 2
    flux_TM = np.linalg.norm(d_minus[neq_PW:neq_PW + num_prop_in]) ** 2
    down_fluxes.append(flux_TE + flux_TM)
    d_plus = rnet_list[-1] @ d_minus
    vec_coef_down.append(d_minus)
    vec_coef_up.append(d_plus)
    flux_TE = np.linalg.norm(d_plus[0:num_prop_in]) ** 2
    flux_TM = np.linalg.norm(d_plus[neq_PW:neq_PW + num_prop_in]) ** 2
    up_flux.append(flux_TE + flux_TM)
    f1_minus = inv_t21_list[-1] @ d_minus
    for i in range(nl - 2):
        f1_plus = rnet_list[-2 * i - 2] @ f1_minus
        f_mat = np.concatenate((f1_minus, f1_plus))
        flux = (f_mat.conj().T @ U_mat @ f_mat)[0, 0]
        down_fluxes.append(flux)
        f2_minus = inv_t12_list[-i - 1] @ f1_minus
        f2_plus = rnet_list[-2 * i - 3] @ P_list[-i - 1] @ f2_minus
        vec_coef_down.append(f2_minus)
        vec_coef_up.append(f2_plus)
        f1_minus = inv_t21_list[-i - 2] @ P_list[-i - 1] @ f2_minus
    f1_plus = rnet_list[0] @ f1_minus
    f2_minus = tnet_list[0] @ f1_minus
    vec_coef_down.append(f2_minus)

    out.warnings = []
    if layers[0].kind == 'film':
        num_prop_out = layers[0].num_prop_pw_per_pol
        if num_prop_out != 0:
            flux_TE = np.linalg.norm(f2_minus[0:num_prop_out]) ** 2
            flux_TM = np.linalg.norm(f2_minus[neq_PW:neq_PW + num_prop_out]) ** 2
            down_fluxes.append(flux_TE + flux_TM)
        else:
            out.warnings.append('no propagating modes in the substrate')
        if num_prop_out != 0:
            a_list, t_list, r_list = _flux_lists(down_fluxes, up_flux, film_substrate=True)
        else:
            a_list = np.zeros(nl - 2)
            r_list = np.zeros(nl - 2)
            t_list = np.zeros(nl - 2)
    else:
        a_list, t_list, r_list = _flux_lists(down_fluxes, up_flux, film_substrate=False)

    out.a_list, out.t_list, out.r_list = a_list, t_list, r_list
    out.vec_coef_down, out.vec_coef_up = vec_coef_down, vec_coef_up
    out.down_fluxes, out.up_flux = down_fluxes, up_flux
    out.inv_t21_list, out.inv_t12_list, out.P_list = inv_t21_list, inv_t12_list, P_list
    return out


def flux_weight_matrix(PW_pols, num_prop_air):
    """The 2P x 2P flux weight U (stack.py:311-321)."""
    neq_PW = PW_pols // 2
    U = np.zeros((2 * PW_pols, 2 * PW_pols), complex)
    for i in range(0, num_prop_air):
        U[i, i] = 1.0
        U[neq_PW + i, neq_PW + i] = 1.0
        U[PW_pols + i, PW_pols + i] = -1.0
        U[PW_pols + neq_PW + i, PW_pols + neq_PW + i] = -1.0
    for i in range(num_prop_air, neq_PW):
        U[i, PW_pols + i] = -1.0j
        U[neq_PW + i, PW_pols + neq_PW + i] = 1.0j
        U[PW_pols + i, i] = 1.0j
        U[PW_pols + neq_PW + i, neq_PW + i] = -1.0j
    return U


def _flux_lists(down_fluxes, up_flux, film_substrate):
    """Absorptance / reflectance / transmittance lists (stack.py:368-426)."""
    a_list, r_list, t_list = [], [], []
    for i in range(1, len(down_fluxes) - 1):
        a_list.append(abs(abs(down_fluxes[i]) - abs(down_fluxes[i + 1])))
    a_list.append(abs(down_fluxes[0] - down_fluxes[-1] - up_flux[0]))
    for i in range(1, len(up_flux) - 1):
        r_list.append(abs(up_flux[i]) / abs(down_fluxes[i]))
    r_list.append(abs(up_flux[0] / down_fluxes[0]))
    for i in range(0, len(down_fluxes) - 2):
        if film_substrate:
            t_list.append(abs(abs(down_fluxes[i + 2]) / abs(down_fluxes[i])))
        else:
            t_list.append(abs(down_fluxes[i + 2]) / abs(down_fluxes[i]))
    t_list.append(abs(down_fluxes[-1] / down_fluxes[0]))
    return a_list, t_list, r_list


# ---------------------------------------------------------------------------
# Convenience: a whole thin-film stack at one spectral point
# ---------------------------------------------------------------------------

def film_stack_point(ns, heights_nm, wl_nm, k_pll, period, period_y=None,
                     max_order=2, world_1d=False, pol='TE', losses=None,
                     incoming_amplitudes=None, shears=None):
    """Solve one all-film stack (bottom to top refractive indices ``ns``)."""
    air = make_air_ref(wl_nm, k_pll, period, period_y, max_order, world_1d)
    if losses is None:
        losses = [True] * len(ns)
    layers = []
    for i, (n, loss) in enumerate(zip(ns, losses)):
        h = None if i in (0, len(ns) - 1) else heights_nm[i - 1]
        layers.append(film_layer(n, wl_nm, k_pll, period, air, h, period_y,
                                 max_order, world_1d, loss))
    res = calc_scat(layers, air, period, pol=pol,
                    incoming_amplitudes=incoming_amplitudes, shears=shears,
                    heights_nm=list(heights_nm))
    res.layers = layers
    res.air = air
    return res


# ---------------------------------------------------------------------------
# Materials
# ---------------------------------------------------------------------------

def material_n(spec, wl_nm, loss=True):
    """Refractive index of a material at wl_nm as backend/materials.py:
    131-161 evaluates it (Material.n) with Anallo.n's loss flag
    (backend/mode_calcs.py:186-192): ``spec`` is a scalar index, a table
    [(wl, n)] or [(wl, Re n, Im n)] interpolated by
    scipy.interpolate.interp1d (linear, the reference's call), or the
    three Drude parameters (omega_plasma, omega_gamma, eps_inf)."""
    from scipy.interpolate import interp1d
    spec = np.asarray(spec)
    if spec.shape == ():
        n = spec.item()
    elif spec.shape == (3,):
        wp, wg, eps_inf = spec
        c = 299792458
        # the reference's expression and evaluation order (materials.py:142)
        n = np.sqrt(eps_inf - wp ** 2 / (((2 * np.pi * c) / (wl_nm * 1e-9)) ** 2
                                         + 1j * wg * (2 * np.pi * c) / (wl_nm * 1e-9)))
    else:
        ns = spec[:, 1] if spec.shape[1] == 2 else spec[:, 1] + 1j * spec[:, 2]
        n = interp1d(spec[:, 0], ns)(wl_nm)
    return n if loss else np.real(n)
