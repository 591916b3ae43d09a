"""Loading helpers for the golden fixtures in tests/golden/ (made by
tests/golden/make_golden.py from the EMUstack reference)."""
from __future__ import annotations

import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')

CASES = ('case_0', 'case_1', 'case_2', 'case_3', 'case_4', 'case_5',
         'synth_config1', 'synth_shear', 'films10', 'edge_cases')


def load_raw(name):
    return dict(np.load(os.path.join(GOLDEN, name + '.npz')))


def _split(flat, lens):
    out, o = [], 0
    for n in lens:
        out.append(flat[o:o + n])
        o += n
    return out


def load_points(name):
    """List of per-spectral-point dicts with nested 'layers'."""
    raw = load_raw(name)
    pts = []
    for p in range(int(raw['n_points'])):
        pre = 'p%d_' % p
        d = {k[len(pre):]: v for k, v in raw.items() if k.startswith(pre)}
        nl = int(d['n_layers'])
        layers = []
        for i in range(nl):
            lp = 'lay%d_' % i
            layers.append({k[len(lp):]: v for k, v in d.items() if k.startswith(lp)})
        d['layers'] = layers
        d['pol'] = str(d['pol'])
        for nm in ('vec_coef_down', 'vec_coef_up'):
            d[nm] = _split(d[nm], d[nm + '_len'])
        for L in layers:
            L['kind'] = str(L['kind'])
        pts.append(d)
    return pts, raw


def oracle_point(pt, use_J=True):
    """Rebuild one golden spectral point with the CPU oracle and solve it."""
    from oracle import gsm_oracle as O
    wl = float(pt['wl_nm'])
    kp = np.asarray(pt['k_pll'], dtype=float)
    per = float(pt['period'])
    per_y = float(pt['period_y'])
    mo = int(pt['max_order'])
    w1d = bool(pt['world_1d'])
    air = O.make_air_ref(wl, kp, per, per_y, mo, w1d)
    layers = []
    nl = len(pt['layers'])
    hs = list(np.asarray(pt['heights_nm'], dtype=float))
    for i, L in enumerate(pt['layers']):
        h = None if i in (0, nl - 1) else hs[i - 1]
        if L['kind'] == 'film':
            layers.append(O.film_layer(complex(L['n']), wl, kp, per, air, h, per_y,
                                       mo, w1d, bool(L['loss'])))
        elif use_J and 'J' in L:
            layers.append(O.OracleLayer('struct', L['k_z'], h, J=L['J'], J_dag=L['J_dag']))
        else:
            layers.append(O.OracleLayer('struct', L['k_z'], h,
                                        rt=(L['R12'], L['T12'], L['R21'], L['T21'])))
    inc = pt.get('incoming')
    shears = pt.get('shears')
    if shears is not None:
        shears = [np.asarray(s) for s in shears]
    res = O.calc_scat(layers, air, per, pol=pt['pol'], incoming_amplitudes=inc,
                      shears=shears, heights_nm=hs)
    res.layers = layers
    res.air = air
    return res


def film_inputs(pt):
    """Inputs of an all-film golden point for emustack_b200.films."""
    n = []
    for L in pt['layers']:
        if L['kind'] != 'film':
            return None
        v = complex(L['n'])
        n.append(v if bool(L['loss']) else complex(v.real, 0.0))
    shears = pt.get('shears')
    return dict(wl=float(pt['wl_nm']), k_pll=np.asarray(pt['k_pll'], float), n=np.array(n),
                heights=np.asarray(pt['heights_nm'], float), pol=pt['pol'],
                incoming=pt.get('incoming'), shears=None if shears is None else np.asarray(shears, float),
                period=float(pt['period']), period_y=float(pt['period_y']),
                max_order=int(pt['max_order']), world_1d=bool(pt['world_1d']))


# ---------------------------------------------------------------------------
# closed-form overlap integrals of fields that are polynomials over the cell
# ---------------------------------------------------------------------------

MESHES = ('4testing-600_120.mail', '4testing-940_266_sq.mail')


def reference_mesh(name):
    """One of the reference's own test meshes (tests/golden/*.mail)."""
    from emustack_b200.mesh import Mesh
    return Mesh.from_mail(os.path.join(GOLDEN, name))


def quadratic_fields(mesh, nval, rng):
    """Transverse fields E_x = f_n(x, y), E_y = g_n(x, y) with f_n, g_n random
    complex quadratics over the whole cell, given at each element's six P2
    nodes (vertices, then the midpoints of edges 1-2, 2-3, 3-1 of the
    straight-sided element), in the reference layout [nel][nval][13][3].
    The P2 interpolation on every element is then the quadratic itself.
    Returns (sol, C) with C[n][component][monomial] over 1, x, y, x^2, xy, y^2."""
    x = mesh.x
    tn = mesh.table_nod - 1
    C = rng.standard_normal((nval, 2, 6)) + 1j * rng.standard_normal((nval, 2, 6))
    v = x[tn[:, :3]]
    mids = np.stack([(v[:, 0] + v[:, 1]) / 2, (v[:, 1] + v[:, 2]) / 2, (v[:, 2] + v[:, 0]) / 2], 1)
    nodes = np.concatenate([v, mids], 1)
    X, Y = nodes[..., 0], nodes[..., 1]
    mon = np.stack([np.ones_like(X), X, Y, X * X, X * Y, Y * Y], -1)
    sol = np.zeros((mesh.nel, nval, 13, 3), complex)
    sol[:, :, :6, 0] = np.einsum('ejm,nm->enj', mon, C[:, 0])
    sol[:, :, :6, 1] = np.einsum('ejm,nm->enj', mon, C[:, 1])
    return sol, C


def exact_J(C, px, py, bloch, d, dy, box, index_pw_inv):
    """J of the quadratic fields over the rectangle box = (x0, x1, y0, y1):
    J_E[s] = (beta I_f - alpha I_g)/|k|, J_K[s] = (alpha I_f + beta I_g)/|k|
    with I_f = int f exp(-i (alpha x + beta y)) dx dy (J_overlap.f:117-198
    integrated exactly): the cell integral factorises into 1D moments
    int x^a exp(-i alpha x) dx, evaluated by 80-point Gauss-Legendre, exact
    to rounding for the orders tested (|alpha| < 60)."""
    x0, x1, y0, y1 = box
    t, w = np.polynomial.legendre.leggauss(80)
    X, WX = 0.5 * (x0 + x1) + 0.5 * (x1 - x0) * t, 0.5 * (x1 - x0) * w
    Y, WY = 0.5 * (y0 + y1) + 0.5 * (y1 - y0) * t, 0.5 * (y1 - y0) * w
    npw, nval = len(px), C.shape[0]
    J = np.zeros((2 * npw, nval), complex)
    for s in range(npw):
        a = bloch[0] + 2 * np.pi / d * px[s]
        b = bloch[1] + 2 * np.pi / dy * py[s]
        mx = np.array([np.sum(WX * X ** k * np.exp(-1j * a * X)) for k in range(3)])
        my = np.array([np.sum(WY * Y ** k * np.exp(-1j * b * Y)) for k in range(3)])
        M = np.array([mx[0] * my[0], mx[1] * my[0], mx[0] * my[1], mx[2] * my[0], mx[1] * my[1],
                      mx[0] * my[2]])
        If, Ig = C[:, 0] @ M, C[:, 1] @ M
        nrm = 1 / np.sqrt(a * a + b * b)
        r = index_pw_inv[s]
        J[r] = (b * If - a * Ig) * nrm
        J[r + npw] = (a * If + b * Ig) * nrm
    return J


# bound on |J_quadrature - J_exact| / max |J_exact| of the 16-point rule on
# the two reference meshes, by max order (measured: 8e-15, 2e-12, 1e-10,
# 1.1e-8 on the 518-triangle mesh)
QUAD_BOUND = {1: 1e-13, 2: 1e-11, 3: 5e-10, 5: 5e-8}
