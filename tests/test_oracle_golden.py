"""Pin the CPU oracle (oracle/gsm_oracle.py) against the EMUstack reference.

Three kinds of golden data, all made by tests/golden/make_golden.py:

* the reference's own outputs re-run in this repository's build container
  (``R_net``, ``T_net``, lists, per-layer interfaces);
* the reference's stored results from its original environment
  (tests/ref/case_N.npz, kept as ``stored_*``), compared at the reference's
  own test tolerance, rtol = atol = 1e-6 (tests/test_case_0_thin_film_multistack.py:142-158);
* the reference's txt spectra (tests/ref/case_N/*.txt, ``txt_*``), compared
  at the reference's tolerances (1e-6; case 3 uses rtol 1e-3 / atol 1e-1,
  tests/test_case_3_simple_mk_msh.py:81-86).
"""
import numpy as np
import pytest

from fixtures import CASES, load_points, oracle_point

TIGHT = dict(rtol=1e-9, atol=1e-11)


@pytest.mark.parametrize('name', CASES)
def test_oracle_matches_reference_run(name):
    pts, raw = load_points(name)
    for p, pt in enumerate(pts):
        res = oracle_point(pt)
        np.testing.assert_allclose(res.R_net, pt['R_net'], **TIGHT, err_msg='%s p%d R_net' % (name, p))
        np.testing.assert_allclose(res.T_net, pt['T_net'], **TIGHT, err_msg='%s p%d T_net' % (name, p))
        np.testing.assert_allclose(np.asarray(res.a_list, float), pt['a_list'], **TIGHT)
        np.testing.assert_allclose(np.asarray(res.t_list, float), pt['t_list'], **TIGHT)
        np.testing.assert_allclose(np.asarray(res.r_list, float), pt['r_list'], **TIGHT)
        for i, (L, (R12, T12, R21, T21)) in enumerate(zip(pt['layers'], res.interfaces)):
            for nm, m in (('R12', R12), ('T12', T12), ('R21', R21), ('T21', T21)):
                np.testing.assert_allclose(m, L[nm], **TIGHT, err_msg='%s p%d lay%d %s' % (name, p, i, nm))
            np.testing.assert_allclose(res.layers[i].k_z, L['k_z'], **TIGHT)
        for a, b in zip(res.vec_coef_down, pt['vec_coef_down']):
            np.testing.assert_allclose(np.ravel(a), b, **TIGHT)
        for a, b in zip(res.vec_coef_up, pt['vec_coef_up']):
            np.testing.assert_allclose(np.ravel(a), b, **TIGHT)


@pytest.mark.parametrize('name', ['case_0', 'case_1', 'case_2', 'case_3', 'case_4', 'case_5'])
def test_oracle_matches_stored_goldens(name):
    """R_net / T_net against the reference's stored npz (its own tolerance, 1e-6)."""
    pts, raw = load_points(name)
    for p, pt in enumerate(pts):
        res = oracle_point(pt)
        np.testing.assert_allclose(res.R_net, raw['p%d_stored_R_net' % p], rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(res.T_net, raw['p%d_stored_T_net' % p], rtol=1e-6, atol=1e-6)
        if name == 'case_0':
            for i in range(len(pt['layers'])):
                for m in ('R12', 'T12', 'R21', 'T21'):
                    np.testing.assert_allclose(res.interfaces[i][('R12', 'T12', 'R21', 'T21').index(m)],
                                               raw['p%d_stored_lay%d_%s' % (p, i, m)], rtol=1e-6, atol=1e-6)
                np.testing.assert_allclose(res.layers[i].k_z, raw['p%d_stored_lay%d_k_z' % (p, i)],
                                           rtol=1e-6, atol=1e-6)


def _txt_columns(res_list, nl):
    """Per-layer spectra in the layout of backend/plotting.py:775-809."""
    a = np.array([[float(v) for v in r.a_list] for r in res_list])
    t = np.array([[float(v) for v in r.t_list] for r in res_list])
    rr = np.array([[float(v) for v in r.r_list] for r in res_list])
    return a, t, rr


@pytest.mark.parametrize('name', ['case_0', 'case_1', 'case_2', 'case_3', 'case_4'])
def test_oracle_matches_txt_spectra(name):
    pts, raw = load_points(name)
    res = [oracle_point(pt) for pt in pts]
    a, t, r = _txt_columns(res, len(pts[0]['layers']))
    rtol, atol = (1e-3, 1e-1) if name == 'case_3' else (1e-6, 1e-6)
    nlay = a.shape[1]
    for key, val in raw.items():
        if not key.startswith('txt_'):
            continue
        fn = key[4:]
        if fn.startswith('Absorptance'):
            col = a[:, nlay - 1]
        elif fn.startswith('Transmittance'):
            col = t[:, nlay - 1]
        elif fn.startswith('Reflectance'):
            col = r[:, -1]
        elif fn.startswith('Lay_Absorb_'):
            col = a[:, int(fn.split('_')[2])]
        elif fn.startswith('Lay_Trans_'):
            col = t[:, int(fn.split('_')[2])]
        else:
            continue
        # the txt files are written with %18.11f
        np.testing.assert_allclose(np.round(col, 11), val[:, 1], rtol=rtol, atol=atol, err_msg=fn)


def test_oracle_interfaces_against_reference():
    from oracle import gsm_oracle as O
    from fixtures import load_raw
    raw = load_raw('interfaces')
    for q in range(int(raw['n_shapes'])):
        out = O.r_t_mat_tf_ns(raw['q%d_Z_air' % q], raw['q%d_J' % q], raw['q%d_J_dag' % q])
        for nm, m in zip(('R12', 'T12', 'R21', 'T21'), out):
            np.testing.assert_allclose(m, raw['q%d_%s' % (q, nm)], **TIGHT)


def test_wood_anomaly_branch_taken():
    pts, raw = load_points('edge_cases')
    res = oracle_point(pts[2])
    assert res.air.wood_anomaly
    np.testing.assert_allclose(res.air.k_z, raw['p2_air_kz'], **TIGHT)
