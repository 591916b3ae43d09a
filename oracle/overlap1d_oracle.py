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

* plane-wave order of a 1D grating          backend/fortran/pw_ordering_1d.f:1-80,
                                            backend/fortran/z_indexx.f:1-105
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


def z_indexx(keys):
    """Ascending index sort of ``keys`` by the algorithm of the reference's
    z_indexx.f:1-105: Numerical Recipes' indexx (Press et al., Numerical
    Recipes, 2nd ed., section 8.4), a median-of-three quicksort with straight
    insertion below 7 elements and an explicit stack.  The order it gives
    tied keys is part of the reference's result, so its steps are followed
    one for one (1-based positions as in the Fortran).  Returns 0-based
    indices."""
    keys = [float(k) for k in keys]
    n, M, NSTACK = len(keys), 7, 50
    indx = list(range(1, n + 1))

    def a0(p):
        return keys[indx[p - 1] - 1]

    def swap(p, q):
        indx[p - 1], indx[q - 1] = indx[q - 1], indx[p - 1]

    istack = [0] * (NSTACK + 1)
    jstack, l, ir = 0, 1, n
    while True:
        if ir - l < M:
            for j in range(l + 1, ir + 1):
                indxt = indx[j - 1]
                a = keys[indxt - 1]
                i = j - 1
                while i >= l:
                    if keys[indx[i - 1] - 1] <= a:
                        break
                    indx[i] = indx[i - 1]
                    i -= 1
                indx[i] = indxt
            if jstack == 0:
                return np.array(indx, dtype=np.int64) - 1
            ir, l = istack[jstack], istack[jstack - 1]
            jstack -= 2
        else:
            k = (l + ir) // 2
            swap(k, l + 1)
            if a0(l) > a0(ir):
                swap(l, ir)
            if a0(l + 1) > a0(ir):
                swap(l + 1, ir)
            if a0(l) > a0(l + 1):
                swap(l, l + 1)
            i, j = l + 1, ir
            indxt = indx[l]
            a = keys[indxt - 1]
            while True:
                i += 1
                while a0(i) < a:
                    i += 1
                j -= 1
                while a0(j) > a:
                    j -= 1
                if j < i:
                    break
                swap(i, j)
            indx[l] = indx[j - 1]
            indx[j - 1] = indxt
            jstack += 2
            if jstack > NSTACK:
                raise RuntimeError('NSTACK too small in indexx')
            if ir - i + 1 >= j - l:
                istack[jstack], istack[jstack - 1] = ir, i
                ir = j - 1
            else:
                istack[jstack], istack[jstack - 1] = j - 1, l
                l = i


def pw_sort_keys(k0, alpha, beta):
    """-Re(kz^2) with kz = sqrt(k0^2 - alpha^2 - beta^2) taken as a complex
    root and squared in complex arithmetic (pw_ordering_1d.f:64-69,
    z_indexx.f:26-28)."""
    z = (k0 ** 2 - np.asarray(alpha, float) ** 2) - np.asarray(beta, float) ** 2
    kz = np.sqrt(np.asarray(z, float).astype(complex))
    return -(kz * kz).real


def pw_order_1d(max_order, period_x, bloch_x, bloch_y, k0):
    """(px, index_pw_inv): the orders px = -max_order..max_order and, for each,
    its 0-based position in the sorted order (pw_ordering_1d.f:53-78: the
    keys -Re(kz^2) ranked by z_indexx)."""
    px = np.arange(-max_order, max_order + 1)
    alpha = bloch_x + 2 * PI / period_x * px
    index_pw = z_indexx(pw_sort_keys(k0, alpha, np.full(len(px), bloch_y)))
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
    pxs, pys, al, be, to_2d = [], [], [], [], np.zeros(npw1, int)
    vec_k = 2 * PI / period_x
    for p in range(-max_order, max_order + 1):
        for q in range(-max_order, max_order + 1):
            if (p / period_x) ** 2 + (q / period_x) ** 2 <= (max_order / period_x) ** 2:
                al.append(bloch_x + vec_k * p)
                be.append(bloch_y + vec_k * q)
                if q == 0:
                    to_2d[p + max_order] = len(pxs)
                pxs.append(p)
                pys.append(q)
    npw2 = len(pxs)
    index_pw_2d = z_indexx(pw_sort_keys(k0, np.array(al), np.array(be)))
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


# ---------------------------------------------------------------------------
# Orthogonality and normalisation of the 1D Bloch modes
# ---------------------------------------------------------------------------

def element_matrices_1d(xmin, xmax):
    """The element matrices orthogonal_1d.f uses (matrix_mxx_1d.f,
    matrix_myy_1d.f, matrix_kxy_1d.f): P2 mass, P3 mass and
    int phi_P2 dpsi_P3/dx, in the reference's rational form."""
    h = xmax - xmin
    mxx = np.array([[4, -1, 2], [-1, 4, 2], [2, 2, 16]], float) * h / 30
    myy = np.array([[128, 19, 99, -36], [19, 128, -36, 99], [99, -36, 648, -81],
                    [-36, 99, -81, 648]], float) * h / 1680
    kxy = np.array([[-83, -7, 99, -9], [7, 83, 9, -99], [-44, 44, -108, 108]], float) / 120
    return mxx, myy, kxy


def overlap_matrix_1d(sol1, sol2, beta1, table_nod, type_el, pp, x_p2, k0, bloch_y):
    """<adjoint i | prime j> of orthogonal_1d.f:60-158: per element the
    11 x 11 matrix [[pp Mxx, 0, -pp Kxy], [0, pp Myy, -i bloch_y pp Myy],
    [0, 0, 0]] (rows adjoint Ex, Ey, Ez; columns prime), applied to
    beta1(j) sol1(j), dotted with sol2(i) (no conjugation), over k0."""
    sol1, sol2 = np.asarray(sol1), np.asarray(sol2)
    nel, nval = sol1.shape[0], sol1.shape[1]
    out = np.zeros((nval, nval), complex)
    for iel in range(nel):
        xmin = x_p2[table_nod[iel][0] - 1]
        xmax = x_p2[table_nod[iel][1] - 1]
        mxx, myy, kxy = element_matrices_1d(xmin, xmax)
        p = pp[type_el[iel] - 1]
        m = np.zeros((11, 11), complex)
        m[0:3, 0:3] = p * mxx
        m[3:7, 3:7] = p * myy
        m[0:3, 7:11] = -p * kxy
        m[3:7, 7:11] = -1j * bloch_y * p * myy
        v = sol1[iel] * np.asarray(beta1)[:, None]          # [nval][11]
        out += (sol2[iel] @ m @ v.T) / k0
    return out


def orthogonal_1d(sol1, sol2, beta1, table_nod, type_el, pp, x_p2, k0, bloch_y):
    """orthogonal_1d.f in full: the overlap matrix, the conjugate-pair swap
    loop (:160-215) on the adjoint modes, and the matrix again with the
    swapped adjoints.  Returns (matrix, swapped sol2, pair_warning)."""
    ovl = overlap_matrix_1d(sol1, sol2, beta1, table_nod, type_el, pp, x_p2, k0, bloch_y)
    perm, warn = pair_swap_order_1d(ovl)
    sol2 = np.asarray(sol2)[:, perm]
    ovl = overlap_matrix_1d(sol1, sol2, beta1, table_nod, type_el, pp, x_p2, k0, bloch_y)
    return ovl, sol2, warn


def pair_swap_order_1d(ovl):
    """The conjugate-pair swap loop of orthogonal_1d.f:160-215 over the
    overlap matrix (rows adjoint, columns prime), applied to mode labels:
    a mode j with |<j|j>| <= 1e-7 swaps its adjoint with every later j2
    with |<j2|j>| > 1e-7 (the matrix is not updated in between) and the
    mode after it is skipped.  Returns (adjoint label at each position,
    pair_warning)."""
    nval = ovl.shape[0]
    lab = list(range(nval))
    j, skip, warn = 0, 0, 0
    while j < nval:
        if abs(ovl[j, j]) > 1e-7:
            j += 1
        elif skip == 0:
            if j == nval - 1:
                warn += 1
            for j2 in range(j + 1, nval):
                if abs(ovl[j2, j]) > 1e-7:
                    lab[j], lab[j2] = lab[j2], lab[j]
            skip = 1
            j += 1
        else:
            skip = 0
            j += 1
    return np.array(lab), warn


def normalise_1d(sol1, sol2, ovl):
    """normalisation_1d.f:15-31: prime and adjoint mode m both divided by
    sqrt(<m|m>) where that root exceeds 1e-8 in magnitude."""
    sol1, sol2 = np.array(sol1, copy=True), np.array(sol2, copy=True)
    for m in range(sol1.shape[1]):
        z = np.sqrt(complex(ovl[m, m]))
        if abs(z) > 1e-8:
            sol1[:, m] /= z
            sol2[:, m] /= z
    return sol1, sol2
