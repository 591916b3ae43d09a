"""CPU oracle for the fields reconstructed from GSM amplitudes.

TEST INFRASTRUCTURE ONLY: a numpy restatement used as the checker by
``tests/``; the product package ``emustack_b200`` never imports it.

Paths are relative to the EMUstack source tree:

* plane-wave fields in a homogeneous layer   backend/plotting.py:2857-2996 (field_values),
                                             backend/plotting.py:1759-1833 (fields_in_plane,
                                             ThinFilm branch)
* x-z slices through ThinFilm layers         backend/plotting.py:2380-2505 (fields_vertically)
* Bloch-mode fields at the P2 nodes of a     backend/fortran/field_value_plane.f:6-132
  2D nanostructured layer

The plane-wave part is pinned against the reference itself: its
``field_values`` run on reference-solved stacks (``tests/golden/fields.npz``,
made by ``tests/golden/make_fields_golden.py``).  The Bloch-mode part is
parity unpinned against reference outputs (the routine is Fortran, with no
compiler for it in this image); it is pinned by closed-form known answers
instead.
"""
from __future__ import annotations

import numpy as np


def pw_layer_coefs(alphas, betas, sort_order, kz, n, vcd, vcu, world_1d=False):
    """Sorted alpha, beta, gamma and the TE / TM eta coefficients of the down
    and up amplitudes, as backend/plotting.py:2896-2941 forms them."""
    s = np.asarray(sort_order)
    alpha = np.asarray(alphas)[s]
    beta = np.asarray(betas) if world_1d else np.asarray(betas)[s]
    gamma = np.asarray(kz, dtype=complex)
    S = len(gamma)
    vcd = np.asarray(vcd, dtype=complex).ravel()
    vcu = np.zeros(2 * S, complex) if vcu is None else np.asarray(vcu, dtype=complex).ravel()
    norm = np.sqrt(alpha ** 2 + beta ** 2)
    k = np.sqrt(alpha ** 2 + beta ** 2 + gamma ** 2)
    chi_te = np.sqrt((n * gamma) / k)
    chi_tm = np.sqrt((n * k) / gamma)
    e_te = (beta / norm, -1 * alpha / norm, np.zeros(np.size(alpha / norm)))
    e_tm = (alpha / norm, beta / norm, -1 * norm / gamma)
    eta = {}
    for name, v in (('down', vcd), ('up', vcu)):
        te, tm = v[:S], v[S:]
        eta[name] = ([(te * e) / chi_te for e in e_te], [(tm * e) / chi_tm for e in e_tm])
    return alpha, beta, gamma, eta


def pw_field_points(alphas, betas, sort_order, kz, n, vcd, vcu, xyz, height_norm=None,
                    substrate=False, world_1d=False):
    """E_x, E_y, E_z, |E| at points (x, y, z) in units of the period: the
    loop of backend/plotting.py:2950-2977.  ``height_norm`` None stands for a
    'semi_inf' layer; ``substrate`` for lay_interest == 0 (z -> -z, no
    upward amplitudes)."""
    alpha, beta, gamma, eta = pw_layer_coefs(alphas, betas, sort_order, kz, n, vcd,
                                             None if substrate else vcu, world_1d)
    out = np.zeros((3, len(xyz)), complex)
    for i, (x1, y1, z1) in enumerate(xyz):
        if world_1d:
            y1 = 0
        z1 = -1 * z1 if substrate else np.abs(z1)
        if height_norm is None:
            e_dn = np.exp(1j * (alpha * x1 + beta * y1 - gamma * z1))
        else:
            e_dn = np.exp(1j * (alpha * x1 + beta * y1 - gamma * (z1 - height_norm)))
        e_up = np.exp(1j * (alpha * x1 + beta * y1 + gamma * z1))
        for c in range(3):
            te = np.sum(eta['down'][0][c] * e_dn + eta['up'][0][c] * e_up)
            tm = np.sum(eta['down'][1][c] * e_dn + eta['up'][1][c] * e_up)
            out[c, i] = te + tm
    tot = np.sqrt(out[0] * np.conj(out[0]) + out[1] * np.conj(out[1]) + out[2] * np.conj(out[2]))
    return out[0], out[1], out[2], tot


def pw_field_grid(alphas, betas, sort_order, kz, n, vcd, vcu, xs, ys, zs, height_norm=None,
                  substrate=False, world_1d=False):
    """Fields on the grid xs x ys x zs, arrays indexed [x, y, z] as
    fields_in_plane builds them (backend/plotting.py:1815-1833; y is not
    zeroed for 1D worlds there)."""
    pts = [(x, y, z) for x in xs for y in ys for z in zs]
    alpha, beta, gamma, eta = pw_layer_coefs(alphas, betas, sort_order, kz, n, vcd,
                                             None if substrate else vcu, world_1d)
    out = np.zeros((3, len(pts)), complex)
    for i, (x1, y1, z1) in enumerate(pts):
        z1 = -1 * z1 if substrate else np.abs(z1)
        dz = z1 if height_norm is None else z1 - height_norm
        e_dn = np.exp(1j * (alpha * x1 + beta * y1 - gamma * dz))
        e_up = np.exp(1j * (alpha * x1 + beta * y1 + gamma * z1))
        for c in range(3):
            out[c, i] = (np.sum(eta['down'][0][c] * e_dn + eta['up'][0][c] * e_up)
                         + np.sum(eta['down'][1][c] * e_dn + eta['up'][1][c] * e_up))
    shape = (len(xs), len(ys), len(zs))
    return tuple(o.reshape(shape) for o in out)


def bloch_field_plane(sol, beta, vec_coef, h, hz):
    """m_E[el, node, component] of field_value_plane
    (backend/fortran/field_value_plane.f:104-130): modes summed in order.
    ``sol`` is C [nel][M][13][3] (Fortran sol(3, 13, M, nel))."""
    sol = np.asarray(sol)
    nel, M = sol.shape[0], sol.shape[1]
    vec_coef = np.asarray(vec_coef, complex).ravel()
    if hz < 0 or hz > h:
        raise ValueError('hz should be in the interval [0, h]')
    mE = np.zeros((nel, 6, 3), complex)
    for m in range(M):
        p_dn = np.exp(1j * beta[m] * hz)
        p_up = np.exp(1j * beta[m] * (h - hz))
        c_dn = vec_coef[m] * p_dn
        c_up = vec_coef[m + M] * p_up
        c_t = c_up + c_dn
        c_z = (c_up - c_dn) / beta[m]
        mE[:, :, 0:2] += sol[:, m, 0:6, 0:2] * c_t
        mE[:, :, 2] += sol[:, m, 0:6, 2] * c_z
    return mE


def vertical_slice(alphas, betas, sort_order, kz, n, vcd, vcu, x_range, z_range, h_norm=None,
                   world_1d=False):
    """E_x, E_y, E_z on the x-z slice at y = 0 of one ThinFilm layer as
    fields_vertically evaluates it (backend/plotting.py:2380-2505): z_range
    as that routine builds it (negative inside the substrate), the down
    term exp(-i gamma z) in the substrate and superstrate (h_norm None) and
    exp(-i gamma (z - h)) in a finite layer; vcu None for the substrate and
    vcd zero for the superstrate without the incoming field.  Arrays
    [x, z]."""
    alpha, beta, gamma, eta = pw_layer_coefs(alphas, betas, sort_order, kz, n, vcd, vcu, world_1d)
    out = np.zeros((3, len(x_range), len(z_range)), complex)
    y1 = 0.0
    for iz, z in enumerate(z_range):
        for ix, x1 in enumerate(x_range):
            if h_norm is None:
                e_dn = np.exp(1j * (alpha * x1 + beta * y1 - gamma * z))
            else:
                e_dn = np.exp(1j * (alpha * x1 + beta * y1 - gamma * (z - h_norm)))
            e_up = np.exp(1j * (alpha * x1 + beta * y1 + gamma * z))
            for c in range(3):
                out[c, ix, iz] = (np.sum(eta['down'][0][c] * e_dn + eta['up'][0][c] * e_up)
                                  + np.sum(eta['down'][1][c] * e_dn + eta['up'][1][c] * e_up))
    return out[0], out[1], out[2]


# the E_y / E_z value at an element's middle from its four P3 values
# (x_min, x_max, h/3, 2h/3): array_sol_P2_1d.f:20-40
P3_MID = np.array([-1.0 / 16.0, -1.0 / 16.0, 9.0 / 16.0, 9.0 / 16.0])


def vertical_slice_1d(sol1, k_z, vec_coef, h_norm, z_range):
    """E_x, E_y, E_z [2 nel + 1][len(z_range)] of a 1D grating layer as
    fields_vertically assembles them (backend/plotting.py:2244-2282): the
    P2 values of array_sol_P2_1d.f per element (x_min, x_max, middle), placed
    in the slice as the routine's loop places them (entry 0 the first
    element's x_min value, then per element its x_max value and its middle
    value), each Bloch mode weighted by vec_coef_down e^{i beta (h - z)} +
    vec_coef_up e^{i beta z} (E_z: the difference over beta).  ``sol1`` is
    [nel][M][11]; ``vec_coef`` the 2M down-then-up amplitudes."""
    sol1 = np.asarray(sol1)
    nel, M = sol1.shape[0], sol1.shape[1]
    vc = np.asarray(vec_coef, complex).ravel()
    out = []
    for comp in range(3):
        if comp == 0:
            p2 = sol1[:, :, 0:3]
        else:
            lo = 3 if comp == 1 else 7
            p2 = np.stack([sol1[:, :, lo], sol1[:, :, lo + 1], sol1[:, :, lo:lo + 4] @ P3_MID], axis=2)
        E = np.zeros((2 * nel + 1, len(z_range)), complex)
        for bm in range(M):
            beta = k_z[bm]
            for h, hz in enumerate(z_range):
                cd = vc[bm] * np.exp(1j * beta * (h_norm - hz))
                cu = vc[bm + M] * np.exp(1j * beta * hz)
                c = (cu - cd) / beta if comp == 2 else cu + cd
                E[0, h] += p2[0, bm, 0] * c
                E[1::2, h] += p2[:, bm, 1] * c      # element x: entry 2x + 1
                E[2::2, h] += p2[:, bm, 2] * c      # element x: entry 2x + 2
        out.append(E)
    return tuple(out)
