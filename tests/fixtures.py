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
