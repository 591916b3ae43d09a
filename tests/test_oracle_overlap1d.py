"""Known-answer tests of the 1D-grating overlap oracle (oracle/overlap1d_oracle.py).

No stored reference result holds J of a 1D layer, so the oracle is pinned by:
* its element integrals against the closed forms of the reference's element
  routines (backend/fortran/vector_p2_exp_1d.f, vector_p3_exp_1d.f), both the
  exact branch and the Taylor branch it takes for |alpha h| <= 1e-3;
* closed-form integrals of constant and linear fields over a whole cell;
* J dagger = conj(J)^T for real fields (the two routines differ only in the
  sign of the exponent, J_overlap_1d.f:175 vs J_dagger_overlap_1d.f:166);
* invariance under element renumbering;
* the embedding in the 2D order set landing on the (px, 0) orders.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import gsm_oracle as G  # noqa: E402
from oracle import overlap1d_oracle as O  # noqa: E402


def _ref_p2(xmin, xmax, alpha):
    """Closed forms of vector_p2_exp_1d.f (int L_i exp(i alpha x))."""
    ah = alpha * (xmax - xmin)
    z1, z2 = np.exp(1j * alpha * xmin), np.exp(1j * alpha * xmax)
    if abs(ah) > 1e-3:
        v = np.array([1j * (-4 + ah ** 2 - 3 * ah * 1j) * z1 + (ah + 4j) * z2,
                      (ah - 4j) * z1 - 1j * (-4 + ah ** 2 + 3 * ah * 1j) * z2,
                      -4 * (2j * (-z1 + z2) + ah * (z1 + z2))])
        return v / (alpha ** 3 * (xmax - xmin) ** 2)
    z3 = np.exp(1j * alpha * (xmax + xmin) / 2)
    v = np.array([(20 + ah ** 2) * z1, (20 + ah ** 2) * z2, -2 * (-40 + ah ** 2) * z3])
    return v / (120 / (xmax - xmin))


def _ref_p3(xmin, xmax, alpha):
    """Closed forms of vector_p3_exp_1d.f."""
    ah = alpha * (xmax - xmin)
    z1, z2 = np.exp(1j * alpha * xmin), np.exp(1j * alpha * xmax)
    if abs(ah) > 1e-3:
        v = np.array([
            (-54 + 11 * ah ** 2 - 36 * ah * 1j + 2 * ah ** 3 * 1j) * z1
            - 2 * (-27 + ah ** 2 + 9 * ah * 1j) * z2,
            -2 * (-27 + ah ** 2 - 9 * ah * 1j) * z1
            + (-54 + 11 * ah ** 2 + 36 * ah * 1j - 2 * ah ** 3 * 1j) * z2,
            9 * (-2 * (-9 + ah ** 2 - 5 * ah * 1j) * z1 + (-18 + ah ** 2 + 8 * ah * 1j) * z2),
            -9 * ((18 - ah ** 2 + 8 * ah * 1j) * z1 + 2 * (-9 + ah ** 2 + 5 * ah * 1j) * z2)])
        return v / (2 * alpha ** 4 * (xmax - xmin) ** 3)
    z3 = np.exp(1j * alpha * (xmax + 2 * xmin) / 3)
    z4 = np.exp(1j * alpha * (2 * xmax + xmin) / 3)
    v = np.array([(30 - ah ** 2 + 4 * ah * 1j) * z1, (30 - ah ** 2 - 4 * ah * 1j) * z2,
                  (90 + ah ** 2 - 12 * ah * 1j) * z3, (90 + ah ** 2 + 12 * ah * 1j) * z4])
    return v / (240 / (xmax - xmin))


@pytest.mark.parametrize('alpha', [-37.0, -6.3, -0.9, 0.05, 2.5, 19.0])
def test_element_integrals_match_the_reference_closed_forms(alpha):
    """The closed forms cancel terms of size up to ~50 down to O((alpha h)^3)
    (P2) and O((alpha h)^4) (P3), so evaluated in a precision with unit
    roundoff u their error is about 500 u h / |alpha h|^3 and / |alpha h|^4.
    They are evaluated here in numpy's extended precision (u ~ 1e-19 on x86;
    the bound loosens by itself where that is plain double), so the oracle's
    quadrature is held to about an ulp of the integrals away from alpha h -> 0."""
    xmin, xmax = 0.13, 0.21
    h = xmax - xmin
    ah = abs(alpha * h)
    u = float(np.finfo(np.longdouble).eps)
    X0, X1, A = np.longdouble(xmin), np.longdouble(xmax), np.longdouble(alpha)
    ref2 = _ref_p2(X0, X1, A).astype(complex)
    ref3 = _ref_p3(X0, X1, A).astype(complex)
    tol2 = 1e-15 + 500 * u * h / ah ** 3
    tol3 = 1e-15 + 500 * u * h / ah ** 4
    np.testing.assert_allclose(O.lagrange_exp_integrals(O.p2_nodes(xmin, xmax), xmin, xmax, alpha),
                               ref2, rtol=0, atol=tol2)
    np.testing.assert_allclose(O.lagrange_exp_integrals(O.p3_nodes(xmin, xmax), xmin, xmax, alpha),
                               ref3, rtol=0, atol=tol3)


def test_element_integrals_small_alpha_branch():
    """Below |alpha h| = 1e-3 the reference switches to a Taylor form; the
    quadrature agrees with it to the Taylor form's own accuracy."""
    xmin, xmax = 0.4, 0.45
    for alpha in (1e-4, -5e-3, 0.0199):
        np.testing.assert_allclose(O.lagrange_exp_integrals(O.p2_nodes(xmin, xmax), xmin, xmax, alpha),
                                   _ref_p2(xmin, xmax, alpha), rtol=0, atol=1e-12)
        np.testing.assert_allclose(O.lagrange_exp_integrals(O.p3_nodes(xmin, xmax), xmin, xmax, alpha),
                                   _ref_p3(xmin, xmax, alpha), rtol=0, atol=1e-12)


def _mesh(nel, seed=0, period=1.0):
    """A P2 mesh of [0, period]: end nodes then midpoints, elements of random
    lengths (x_p2 indices 1-based, as the reference's table_nod)."""
    rng = np.random.default_rng(seed)
    cuts = np.sort(np.concatenate(([0.0, period], rng.uniform(0, period, nel - 1))))
    ends = list(cuts)
    mids = list(0.5 * (cuts[1:] + cuts[:-1]))
    x = np.array(ends + mids)
    tab = np.array([[i + 1, i + 2, len(ends) + i + 1] for i in range(nel)])
    return x, tab


def test_constant_and_linear_fields_over_the_cell():
    """Ex = 1 and Ey = x (both represented exactly by P2 / P3): J's E rows are
    RE . (int exp(-i a x), int x exp(-i a x)) over the cell."""
    period, max_order, bx, by, k0 = 1.0, 3, 0.7, 0.4, 9.0
    x, tab = _mesh(7, seed=1, period=period)
    nel = len(tab)
    sol = np.zeros((nel, 1, 11), complex)
    for e in range(nel):
        xmin, xmax = x[tab[e][0] - 1], x[tab[e][1] - 1]
        sol[e, 0, 0:3] = 1.0
        sol[e, 0, 3:7] = O.p3_nodes(xmin, xmax)
    px, inv = O.pw_order_1d(max_order, period, bx, by, k0)
    J = O.overlap_1d(sol, tab, x, period, bx, by, max_order, inv)
    npw = len(px)
    for o in range(npw):
        a = bx + 2 * np.pi * px[o] / period
        i0 = (np.exp(-1j * a * period) - 1) / (-1j * a)
        i1 = (np.exp(-1j * a * period) * (1j * a * period + 1) - 1) / (a * a)  # int_0^d x e^{-iax}
        norm = 1 / np.hypot(a, by)
        re, rk = np.array([by, -a]) * norm, np.array([a, by]) * norm
        np.testing.assert_allclose(J[inv[o], 0], re[0] * i0 + re[1] * i1, rtol=1e-10, atol=1e-13)
        np.testing.assert_allclose(J[inv[o] + npw, 0], rk[0] * i0 + rk[1] * i1, rtol=1e-10, atol=1e-13)


def test_dagger_is_conjugate_transpose_for_real_fields_and_renumbering_invariance():
    period, max_order, bx, by, k0 = 1.0, 4, 0.3, 0.0, 12.0
    x, tab = _mesh(9, seed=2, period=period)
    rng = np.random.default_rng(3)
    sol = rng.normal(size=(len(tab), 5, 11)) + 0j
    px, inv = O.pw_order_1d(max_order, period, bx, by, k0)
    J = O.overlap_1d(sol, tab, x, period, bx, by, max_order, inv)
    Jd = O.overlap_1d(sol, tab, x, period, bx, by, max_order, inv, dagger=True)
    np.testing.assert_allclose(Jd, J.conj().T, rtol=1e-12, atol=1e-14)
    perm = rng.permutation(len(tab))
    J2 = O.overlap_1d(sol[perm], tab[perm], x, period, bx, by, max_order, inv)
    np.testing.assert_allclose(J2, J, rtol=1e-12, atol=1e-14)


def test_plane_wave_order_matches_the_air_sort():
    """The 1D order is the air's -Re k_z + Im k_z order over px (1D grating)."""
    period, max_order, wl = 600.0, 5, 700.0
    kp = G.k_parallel_from_angles(wl, 0.2, 0.0)
    air = G.make_air_ref(wl, kp, period, None, max_order, world_1d=True)
    k0 = 2 * np.pi / G.wl_norm(wl, period)
    bx, by = kp * period
    px, inv = O.pw_order_1d(max_order, 1.0, bx, by, k0)
    np.testing.assert_array_equal(px[np.argsort(inv)], air.pxs[air.sort_order])


def test_embedding_in_the_2d_order_set():
    """Each 1D order px lands, for J and J dagger, at the sorted position of
    the 2D order (px, 0); every other row (column) is zero."""
    period, max_order, bx, by, k0 = 1.0, 3, 0.5, 0.2, 8.0
    x, tab = _mesh(5, seed=4, period=period)
    rng = np.random.default_rng(5)
    sol = rng.normal(size=(len(tab), 3, 11)) + 1j * rng.normal(size=(len(tab), 3, 11))
    px, inv = O.pw_order_1d(max_order, period, bx, by, k0)
    J = O.overlap_1d(sol, tab, x, period, bx, by, max_order, inv)
    Jd = O.overlap_1d(sol, tab, x, period, bx, by, max_order, inv, dagger=True)
    J2, Jd2, (p2, q2) = O.pw_matrix_1d_to_2d(J, Jd, period, bx, by, max_order, k0, inv)
    gp, gq = G.grating_orders_2d(max_order, period, period)
    np.testing.assert_array_equal(p2, gp)
    np.testing.assert_array_equal(q2, gq)
    npw1, npw2 = len(px), len(p2)
    kz = np.sqrt((k0 ** 2 - (bx + 2 * np.pi * p2) ** 2 - (by + 2 * np.pi * q2) ** 2).astype(complex))
    pos = np.empty(npw2, int)
    pos[np.argsort(-1 * kz.real + kz.imag, kind='stable')] = np.arange(npw2)
    used = []
    for o in range(npw1):
        s = pos[np.nonzero((p2 == px[o]) & (q2 == 0))[0][0]]
        used += [s, s + npw2]
        np.testing.assert_array_equal(J2[s], J[inv[o]])
        np.testing.assert_array_equal(J2[s + npw2], J[inv[o] + npw1])
        np.testing.assert_array_equal(Jd2[:, s], Jd[:, inv[o]])
        np.testing.assert_array_equal(Jd2[:, s + npw2], Jd[:, inv[o] + npw1])
    rest = np.setdiff1d(np.arange(2 * npw2), used)
    assert not J2[rest].any() and not Jd2[:, rest].any()


def test_z_indexx_hand_traced_ties():
    """The reference ranks plane waves with Numerical Recipes' indexx
    (z_indexx.f).  For px = -4..4 at zero Bloch vector the keys are
    alpha^2 - k0^2 with alpha = 2 pi px, tied in pairs +-px.  Traced by hand
    through its steps (n = 9 > 7: one partition about the median of
    keys(1), keys(5), keys(9), which leaves positions 1-7 to straight
    insertion and 8-9 in place) the order is px = 0, -1, 1, -2, 2, 3, -3,
    -4, 4: ties are NOT broken by generation index for px = +-3."""
    px, inv = O.pw_order_1d(4, 1.0, 0.0, 0.0, 2 * np.pi / 1.3)
    order = np.empty_like(inv)
    order[inv] = np.arange(len(inv))
    np.testing.assert_array_equal(px[order], [0, -1, 1, -2, 2, 3, -3, -4, 4])


def test_z_indexx_sorts_and_is_stable_below_seven():
    rng = np.random.default_rng(3)
    for t in range(400):
        n = int(rng.integers(1, 70))
        keys = rng.integers(0, 6, n).astype(float) if t % 2 else rng.standard_normal(n)
        idx = O.z_indexx(keys)
        assert sorted(idx.tolist()) == list(range(n))
        assert np.all(np.diff(keys[idx]) >= 0)
        if n < 7:   # straight insertion only: ties keep their input order
            np.testing.assert_array_equal(idx, np.argsort(keys, kind='stable'))


def test_element_matrices_are_the_lagrange_integrals():
    """The GPU kernel forms the element matrices of the 1D orthogonality
    integral from the Lagrange coefficients of the P2 / P3 bases on [0, 1]
    (overlap1d.cu kP2c / kP3c); they equal the reference's rational tables
    (matrix_mxx_1d.f, matrix_myy_1d.f, matrix_kxy_1d.f)."""
    P2 = np.array([[1, -3, 2], [0, -1, 2], [0, 4, -4]], float)
    P3 = np.array([[1, -5.5, 9, -4.5], [0, 1, -4.5, 4.5], [0, 9, -22.5, 13.5], [0, -4.5, 18, -13.5]])
    for node, coef, pts in ((O.p2_nodes, P2, 3), (O.p3_nodes, P3, 4)):
        t = node(0.0, 1.0)
        V = np.vander(t, pts, increasing=True)
        np.testing.assert_allclose(coef @ V.T, np.eye(pts), atol=1e-14)   # l_i(t_j) = delta_ij
    mxx = np.array([[sum(P2[i, p] * P2[j, q] / (p + q + 1) for p in range(3) for q in range(3))
                     for j in range(3)] for i in range(3)])
    myy = np.array([[sum(P3[i, p] * P3[j, q] / (p + q + 1) for p in range(4) for q in range(4))
                     for j in range(4)] for i in range(4)])
    kxy = np.array([[sum(P2[i, p] * q * P3[j, q] / (p + q) for p in range(3) for q in range(1, 4))
                     for j in range(4)] for i in range(3)])
    h = 0.37
    rm, ry, rk = O.element_matrices_1d(0.2, 0.2 + h)
    np.testing.assert_allclose(h * mxx, rm, atol=1e-15)
    np.testing.assert_allclose(h * myy, ry, atol=1e-14)
    np.testing.assert_allclose(kxy, rk, atol=1e-14)


def test_host_pair_swap_matches_the_oracle():
    """The drop-in's host port of the conjugate-pair swap loop
    (emustack_b200.overlap.reorder_pairs_1d) gives the same permutation as
    the oracle's literal restatement, on matrices with vanishing diagonals."""
    from emustack_b200.overlap import reorder_pairs_1d
    rng = np.random.default_rng(8)
    for t in range(60):
        M = int(rng.integers(2, 12))
        ovl = rng.standard_normal((M, M)) + 1j * rng.standard_normal((M, M))
        ovl[rng.random((M, M)) < 0.4] *= 1e-9
        small = rng.random(M) < 0.5
        ovl[np.arange(M)[small], np.arange(M)[small]] = 1e-9
        perm, warn = reorder_pairs_1d(ovl)
        lab, w = O.pair_swap_order_1d(ovl)
        np.testing.assert_array_equal(perm, lab)
        assert warn == w
