"""The film kernels' rewritten recursion against the reference's, on the CPU.

The film kernels (emustack_b200/csrc/film_core.cuh) do not evaluate the
reference's interface and cascade formulas (backend/mode_calcs.py:451-477,
backend/stack.py:229-278) literally: between two air gaps they use impedances
scaled by k_z k_z,air (TE) or k k_air (TM), use T12 T21 + R12^2 = 1 to
write each gap-and-layer step as a Moebius map with one quotient, and fold
the per-layer transmission into x1 p x2 = 4AB p / D over the same
denominator.  This file restates that form in numpy
(vectorised over the orders of one point) and checks it against the oracle's
literal restatement of the reference, so the algebra is pinned without a GPU.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import gsm_oracle as O  # noqa: E402


def kernel_form(ns, heights_nm, wl_nm, k_pll, period, max_order):
    """R_net, T_net diagonals (TE half then TM half) and the per-layer
    products x1 p x2, in the kernels' form."""
    air = O.make_air_ref(wl_nm, k_pll, period, None, max_order)
    wln = O.wl_norm(wl_nm, period)
    kair = 2 * np.pi / wln
    npw = air.num_pw_per_pol
    kz_air = air.k_z[:npw]
    L = len(ns)
    mods = [O.FilmModes(n, wl_nm, k_pll, period, None, max_order, air=air) for n in ns]
    z_air = air.Z()

    def scaled_ab(l):
        m = mods[l]
        k, n, kz = m.k(), m.n_val, m.k_z[:npw]
        A = np.concatenate((k / n * kz_air, kair / n * kz))
        B = np.concatenate((kair * kz, k * kz_air))
        return A, B

    def scaled(l):
        A, B = scaled_ab(l)
        R = (A - B) / (A + B)
        TT = 4 * A * B / (A + B) ** 2
        return R, TT

    def t12(l):
        z2 = mods[l].Z()
        return 2 * np.sqrt(z2) * np.sqrt(z_air) / (z2 + z_air)

    R0, _ = scaled(0)
    rnet, tnet = R0, t12(0)
    g_list = []
    for l in range(1, L - 1):
        # Moebius form: s = A + B, d = A - B, u = s - d r, v = s r - d,
        # D = s u + d p^2 v, N = d u + s p^2 v; r' = N / D, x1 p x2 = 4 A B p / D
        A, B = scaled_ab(l)
        s_, d_ = A + B, A - B
        kz = mods[l].k_z
        p = np.exp(1j * kz * heights_nm[l - 1] / period)
        u = s_ - d_ * rnet
        v = s_ * rnet - d_
        w = p * p * v
        D = s_ * u + d_ * w
        N = d_ * u + s_ * w
        g = 4 * A * B * p / D
        g_list.append(g)
        tnet = tnet * g
        rnet = N / D
    R, TT = scaled(L - 1)
    d1 = 1 / (1 - R * rnet)
    tnet = tnet * t12(L - 1) * d1
    rnet = TT * d1 * rnet - R
    return rnet, tnet, g_list


@pytest.mark.parametrize('seed', range(6))
def test_kernel_form_equals_reference_recursion(seed):
    rng = np.random.default_rng(seed)
    L = int(rng.integers(2, 9))
    ns = list(rng.uniform(1.2, 4.0, L) + 1j * rng.uniform(0.0, 0.4, L))
    ns[-1] = 1.0 + 0j if seed % 2 else ns[-1]
    heights = list(rng.uniform(20, 300, L - 2))
    wl = float(rng.uniform(350, 1100))
    th, ph = rng.uniform(0, 1.0), rng.uniform(0, 1.5)
    kp = O.k_parallel_from_angles(wl, th, ph)
    period, max_order = 500.0, 3
    res = O.film_stack_point(ns, heights, wl, kp, period, max_order=max_order, pol='TE')
    rnet, tnet, _ = kernel_form(ns, heights, wl, kp, period, max_order)
    np.testing.assert_allclose(rnet, np.diag(res.R_net), rtol=1e-11, atol=1e-13)
    np.testing.assert_allclose(tnet, np.diag(res.T_net), rtol=1e-11, atol=1e-13)


def test_transmission_product_is_x1_p_x2():
    """The per-layer product the kernels save for the flux pass equals the
    reference's t21 (I - r12 r)^-1 p t12 (I + r12 p r_gap p)^-1 chain."""
    rng = np.random.default_rng(11)
    L = 6
    ns = list(rng.uniform(1.3, 3.5, L) + 1j * rng.uniform(0.0, 0.3, L))
    heights = list(rng.uniform(30, 250, L - 2))
    wl, period, max_order = 633.0, 500.0, 2
    kp = O.k_parallel_from_angles(wl, 0.3, 0.2)
    _, _, g_list = kernel_form(ns, heights, wl, kp, period, max_order)
    air = O.make_air_ref(wl, kp, period, None, max_order)
    z_air = air.Z()
    mods = [O.FilmModes(n, wl, kp, period, None, max_order, air=air) for n in ns]
    # literal reference quantities, diagonal form
    z0 = mods[0].Z()
    r = (z0 - z_air) / (z0 + z_air)
    for l in range(1, L - 1):
        z2 = mods[l].Z()
        R12 = (z2 - z_air) / (z2 + z_air)
        T12 = 2 * np.sqrt(z2) * np.sqrt(z_air) / (z2 + z_air)
        p = np.exp(1j * mods[l].k_z * heights[l - 1] / period)
        x1 = T12 / (1 - R12 * r)
        rg = -R12 + T12 * r * x1
        x2 = T12 / (1 + R12 * p * rg * p)
        np.testing.assert_allclose(g_list[l - 1], x1 * p * x2, rtol=1e-11, atol=1e-14)
        r = R12 + T12 * p * rg * p * x2


def _sort_key(k):
    """numpy restatement of film_core.cuh sort_key: -0 taken as +0, then the
    sign bit flipped for positive doubles and all bits for negative ones."""
    b = (np.asarray(k, np.float64) + 0.0).view(np.int64)
    u = b.view(np.uint64)
    return np.where(b < 0, ~u, u | np.uint64(1 << 63))


def test_integer_sort_keys_rank_as_the_doubles():
    """The kernels rank orders by -Re k_z + Im k_z with integer keys; the
    ranks (stable on ties) equal those of the double comparison, signed
    zeros and exact ties included."""
    rng = np.random.default_rng(3)
    k = np.concatenate((rng.normal(size=200) * 10.0 ** rng.integers(-300, 300, 200),
                        [0.0, -0.0, 1.0, 1.0, -1.0, -1.0, 5e-324, -5e-324, 1e308, -1e308]))
    rng.shuffle(k)
    keys = _sort_key(k)
    r_int = np.array([np.sum((keys < keys[u]) | ((keys == keys[u]) & (np.arange(len(k)) < u)))
                      for u in range(len(k))])
    r_dbl = np.array([np.sum((k < k[u]) | ((k == k[u]) & (np.arange(len(k)) < u)))
                      for u in range(len(k))])
    np.testing.assert_array_equal(r_int, r_dbl)
    np.testing.assert_array_equal(np.sort(r_int), np.arange(len(k)))


def test_layer_recursion_as_moebius_product():
    """The per-layer step r -> r' of the film recursion is a Moebius map whose
    2 x 2 matrix, with T12 T21 + R12^2 = 1, is [[p^2 - R^2, R(1 - p^2)],
    [R(p^2 - 1), 1 - R^2 p^2]]; the superstrate's gap is [[1, -R], [-R, 1]].
    The product of the matrices applied to (R_substrate, 1) gives R_net, and
    T_net = T12(substrate) prod(T12 T21 p) T12(top) / (second component):
    the form a layer-parallel reduction would evaluate."""
    rng = np.random.default_rng(5)
    for trial in range(4):
        L = int(rng.integers(3, 10))
        ns = list(rng.uniform(1.2, 4.0, L) + 1j * rng.uniform(0.0, 0.4, L))
        heights = list(rng.uniform(20, 300, L - 2))
        wl = float(rng.uniform(400, 1000))
        kp = O.k_parallel_from_angles(wl, rng.uniform(0, 1.0), rng.uniform(0, 1.5))
        period, max_order = 500.0, 2
        res = O.film_stack_point(ns, heights, wl, kp, period, max_order=max_order, pol='TE')
        air = O.make_air_ref(wl, kp, period, None, max_order)
        z_air = air.Z()
        mods = [O.FilmModes(n, wl, kp, period, None, max_order, air=air) for n in ns]
        R = [(m.Z() - z_air) / (m.Z() + z_air) for m in mods]
        T12 = [2 * np.sqrt(m.Z()) * np.sqrt(z_air) / (m.Z() + z_air) for m in mods]
        N, D = R[0].copy(), np.ones_like(R[0])
        tprod = T12[0].copy()
        for l in range(1, L - 1):
            p = np.exp(1j * mods[l].k_z * heights[l - 1] / period)
            u, r = p * p, R[l]
            m00, m01, m10, m11 = u - r * r, r * (1 - u), r * (u - 1), 1 - r * r * u
            N, D = m00 * N + m01 * D, m10 * N + m11 * D
            tprod = tprod * T12[l] * T12[l] * p
        r = R[L - 1]
        N, D = N - r * D, -r * N + D
        np.testing.assert_allclose(N / D, np.diag(res.R_net), rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(tprod * T12[L - 1] / D, np.diag(res.T_net), rtol=1e-10, atol=1e-12)


def _seed(x, bits=16):
    """A seed with only `bits` correct bits: the exact value with its
    mantissa cut to that width and perturbed by up to 2^-bits relative."""
    x = np.asarray(x, np.float64)
    m, e = np.frexp(x)
    m = np.round(m * 2.0 ** bits) / 2.0 ** bits
    rng = np.random.default_rng(1)
    return np.ldexp(m, e) * (1 + rng.uniform(-1, 1, x.shape) * 2.0 ** -bits)


def test_newton_steps_reach_double_precision_from_a_16_bit_seed():
    """emu_fastmath.cuh takes two Newton steps from the hardware's approximate
    reciprocal and reciprocal square root.  From any seed with 16 correct
    bits, two steps land within a few ulps over the range the kernels use
    (numpy rounds the products that the kernels fuse into multiply-adds, so
    the kernels' steps are at least as accurate as these)."""
    rng = np.random.default_rng(0)
    a = 10.0 ** rng.uniform(-290, 290, 20000) * rng.choice([-1.0, 1.0], 20000)
    x = _seed(1.0 / a)
    for _ in range(2):
        e = np.float64(1.0) - a * x          # fma(-a, x, 1) up to the last bit
        x = x + x * e
    assert np.max(np.abs(x * a - 1.0)) < 8 * np.finfo(np.float64).eps
    q = np.abs(a)[np.abs(np.log10(np.abs(a))) < 280]
    y = _seed(1.0 / np.sqrt(q))
    for _ in range(2):
        e = 0.5 - (0.5 * q * y) * y
        y = y + y * e
    assert np.max(np.abs(y * np.sqrt(q) - 1.0)) < 8 * np.finfo(np.float64).eps
