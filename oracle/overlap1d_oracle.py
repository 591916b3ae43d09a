"""CPU oracle for the overlap integrals of 1D-grating layers (J, J dagger).

TEST INFRASTRUCTURE ONLY: a numpy restatement used as the checker by
``tests/``; the product package ``emustack_b200`` never imports it.

Parity unpinned against reference outputs: the reference computes these
integrals in Fortran (no compiler for it in this image) and its stored golden
results hold the 1D layers' interfaces, not their fields or J.  This module is
pinned by known answers instead (``tests/test_oracle_overlap1d.py``), and its
element integrals, which it evaluates by Gauss-Legendre quadrature, are
checked against the closed forms of the reference's element routines.

Paths are relative to the EMUstack source tree:

* plane-wave order of a 1D grating          backend/fortran/pw_ordering_1d.f:1-80
* J  (E rows, then K rows)                  backend/fortran/J_overlap_1d.f:8-200
* J dagger (conjugate plane waves)          backend/fortran/J_dagger_overlap_1d.f:1-225
* element integrals of P2 / P3 x exp        backend/fortran/vector_p2_exp_1d.f,
                                            backend/fortran/vector_p3_exp_1d.f
* embedding in the 2D order set             backend/fortran/pw_matrix_1d_to_2d.f:1-200
* call sequence                             backend/fortran/py_calc_modes_1d.f:583-620

Field layout, as the reference passes it: ``sol`` is Fortran ``(11, nval, nel)``
= C ``[nel][nval][11]``: entries 0-2 Ex at the element's P2 nodes
(x_min, x_max, midpoint), 3-6 Ey at its P3 nodes (x_min, x_max, x_min + h/3,
x_min + 2h/3), 7-10 Ez (not used by J).  ``table_nod`` is ``[nel][3]``, 1-based
indices into ``x_p2`` (first two entries: the element's end nodes).
"""
from __future__ import annotations

import numpy as np

PI = np.pi


def p2_nodes(xmin, xmax):
    """P2 Lagrange nodes of one element, in the reference's local order."""
    return np.array([xmin, xmax, 0.5 * (xmin + xmax)])


def p3_nodes(xmin, xmax):
    """P3 Lagrange nodes of one element, in the reference's local order."""
    h = xmax - xmin
    return np.array([xmin, xmax, xmin + h / 3.0, xmin + 2.0 * h / 3.0])


def lagrange_exp_integrals(nodes, xmin, xmax, alpha):
    """int_{xmin}^{xmax} L_i(x) exp(i alpha x) dx for the Lagrange basis L_i of
    ``nodes``, by Gauss-Legendre quadrature with enough points that the
    polynomial times the exponential is integrated to rounding (the
    reference evaluates the same integrals in closed form)."""
    h = xmax - xmin
    n = 24 + int(np.ceil(abs(alpha) * abs(h)))
    t, w = np.polynomial.legendre.leggauss(n)
    x = 0.5 * (xmin + xmax) + 0.5 * h * t
    w = 0.5 * h * w
    e = np.exp(1j * alpha * x)
    out = np.empty(len(nodes), complex)
    for i, xi in enumerate(nodes):
        li = np.ones_like(x)
        for j, xj in enumerate(nodes):
            if j != i:
                li = li * (x - xj) / (xi - xj)
        out[i] = np.sum(w * li * e)
    return out


def pw_order_1d(max_order, period_x, bloch_x, bloch_y, k0):
    """(px, index_pw_inv): the orders px = -max_order..max_order and, for each,
    its 0-based position in the sorted order (pw_ordering_1d.f: k_z =
    sqrt(k0^2 - alpha^2 - beta^2) sorted by the key -Re k_z + Im k_z, as the
    air's plane waves are sorted, z_indexx.f:22-28)."""
    px = np.arange(-max_order, max_order + 1)
    alpha = bloch_x + 2 * PI / period_x * px
    kz = np.sqrt((k0 ** 2 - alpha ** 2 - bloch_y ** 2).astype(complex))
    index_pw = np.argsort(-1 * kz.real + kz.imag, kind='stable')
    inv = np.empty_like(index_pw)
    inv[index_pw] = np.arange(len(px))
    return px, inv


def _pw_vectors(alpha, bloch_y):
    """Unit transverse vectors of one plane wave (J_overlap_1d.f:146-166):
    RK along (alpha, beta), RE = (beta, -alpha); (0, 1) and (1, 0) at normal
    incidence on the zero order."""
    if alpha != 0.0 or bloch_y != 0.0:
        norm = 1.0 / np.sqrt(alpha ** 2 + bloch_y ** 2)
        return np.array([alpha * norm, bloch_y * norm]), np.array([bloch_y * norm, -alpha * norm])
    return np.array([0.0, 1.0]), np.array([1.0, 0.0])


def overlap_1d(sol, table_nod, x_p2, period_x, bloch_x, bloch_y, max_order, index_pw_inv,
               dagger=False):
    """J (``dagger=False``: plane waves exp(-i alpha x), shape (2 Npw, nval),
    rows E then K) or J dagger (``dagger=True``: exp(+i alpha x), shape
    (nval, 2 Npw)), both with the plane waves at their sorted positions
    (J_overlap_1d.f:130-200, J_dagger_overlap_1d.f:120-222)."""
    sol = np.asarray(sol)
    nel, nval = sol.shape[0], sol.shape[1]
    px = np.arange(-max_order, max_order + 1)
    npw = len(px)
    ovl_k = np.zeros((npw, nval), complex)
    ovl_e = np.zeros((npw, nval), complex)
    sign = 1.0 if dagger else -1.0
    for iel in range(nel):
        xmin = x_p2[table_nod[iel][0] - 1]
        xmax = x_p2[table_nod[iel][1] - 1]
        n2, n3 = p2_nodes(xmin, xmax), p3_nodes(xmin, xmax)
        for o in range(npw):
            s2 = index_pw_inv[o]
            alpha = bloch_x + 2 * PI / period_x * px[o]
            rk, re = _pw_vectors(alpha, bloch_y)
            i2 = lagrange_exp_integrals(n2, xmin, xmax, sign * alpha)
            i3 = lagrange_exp_integrals(n3, xmin, xmax, sign * alpha)
            phi_x = sol[iel, :, 0:3] @ i2
            phi_y = sol[iel, :, 3:7] @ i3
            ovl_k[s2] += phi_x * rk[0] + phi_y * rk[1]
            ovl_e[s2] += phi_x * re[0] + phi_y * re[1]
    J = np.concatenate((ovl_e, ovl_k))
    return J.T.copy() if dagger else J


def pw_matrix_1d_to_2d(J_1d, Jd_1d, period_x, bloch_x, bloch_y, max_order, k0, index_pw_inv_1d):
    """Embed J (2 Npw_1d, nval) and J dagger (nval, 2 Npw_1d) of the 1D order
    set in the 2D order set of the same maximum order, zero elsewhere
    (pw_matrix_1d_to_2d.f): the 2D set takes period_x for both directions,
    each 1D order px goes to the 2D order (px, 0), both at their sorted
    positions."""
    npw1 = 2 * max_order + 1
    pxs, pys, kzs, to_2d = [], [], [], np.zeros(npw1, int)
    vec_k = 2 * PI / period_x
    for p in range(-max_order, max_order + 1):
        for q in range(-max_order, max_order + 1):
            if (p / period_x) ** 2 + (q / period_x) ** 2 <= (max_order / period_x) ** 2:
                a, b = bloch_x + vec_k * p, bloch_y + vec_k * q
                kzs.append(np.sqrt(complex(k0 ** 2 - a ** 2 - b ** 2)))
                if q == 0:
                    to_2d[p + max_order] = len(pxs)
                pxs.append(p)
                pys.append(q)
    kzs = np.array(kzs)
    npw2 = len(kzs)
    index_pw_2d = np.argsort(-1 * kzs.real + kzs.imag, kind='stable')
    inv2 = np.empty_like(index_pw_2d)
    inv2[index_pw_2d] = np.arange(npw2)
    nval = J_1d.shape[1]
    J2 = np.zeros((2 * npw2, nval), complex)
    Jd2 = np.zeros((nval, 2 * npw2), complex)
    for o in range(npw1):
        s1 = index_pw_inv_1d[o]
        s2 = inv2[to_2d[o]]
        J2[s2] = J_1d[s1]
        J2[s2 + npw2] = J_1d[s1 + npw1]
        Jd2[:, s2] = Jd_1d[:, s1]
        Jd2[:, s2 + npw2] = Jd_1d[:, s1 + npw1]
    return J2, Jd2, (np.array(pxs), np.array(pys))
