"""CPU checks of the field oracle and of the data writers.

* The plane-wave field oracle (oracle/fields_oracle.py) reproduces the
  reference's own field_values (backend/plotting.py:2857-2996) on
  reference-solved stacks (tests/golden/fields.npz), and the tangential
  field it gives is continuous across every interface of those stacks.
* The Bloch-mode field oracle (field_value_plane.f) meets closed-form
  answers.
* The text writer (emustack_b200.fields.t_r_a_write_files) writes the
  reference's files byte for byte from the same spectra; the npz writer
  (save_reference_data) keeps the layout of tests/testing.py.
"""
import os
import types

import numpy as np
import pytest

from oracle import fields_oracle as F

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, 'golden', 'fields.npz'))


def _layer_args(key, i):
    d = GOLD
    L = len(d[key + 'n'])
    w1d = bool(d[key + 'world_1d'])
    lk = key + 'lay%d_' % i
    row = L - 1 - i
    h = None if i in (0, L - 1) else d[key + 'heights_nm'][i - 1] / float(d[key + 'period'])
    betas = d[lk + 'betas']
    if w1d and betas.size == 1:
        betas = betas[0]
    return dict(alphas=d[lk + 'alphas'], betas=betas, sort_order=d[lk + 'sort_order'], kz=d[lk + 'kz'],
                n=complex(d[lk + 'n']), vcd=d[key + 'vec_coef_down'][row],
                vcu=None if i == 0 else d[key + 'vec_coef_up'][row], height_norm=h, substrate=(i == 0),
                world_1d=w1d)


def _cases():
    for key in GOLD['names']:
        for i in range(len(GOLD[key + 'n'])):
            yield str(key), i


@pytest.mark.parametrize('key,i', list(_cases()))
def test_pw_oracle_reproduces_the_reference(key, i):
    lk = key + 'lay%d_' % i
    Ex, Ey, Ez, Et = F.pw_field_points(xyz=GOLD[lk + 'xyz'], **_layer_args(key, i))
    ref = GOLD[lk + 'E']
    scale = np.abs(ref).max()
    np.testing.assert_allclose(np.array([Ex, Ey, Ez]), ref, rtol=0, atol=1e-14 * scale)
    np.testing.assert_allclose(Et, GOLD[lk + 'E_tot'], rtol=0, atol=1e-14 * scale)


@pytest.mark.parametrize('key', [str(k) for k in GOLD['names']])
def test_tangential_field_is_continuous_across_interfaces(key):
    """E_x and E_y just below and just above every interface agree: the GSM
    amplitudes and the field formula satisfy the boundary condition."""
    L = len(GOLD[key + 'n'])
    hs = GOLD[key + 'heights_nm'] / float(GOLD[key + 'period'])
    xy = np.random.default_rng(1).uniform(0, 1, (6, 2))
    for i in range(L - 1):
        ztop = 0.0 if i == 0 else hs[i - 1]
        below = F.pw_field_points(xyz=np.column_stack([xy, np.full(6, ztop)]), **_layer_args(key, i))
        above = F.pw_field_points(xyz=np.column_stack([xy, np.zeros(6)]), **_layer_args(key, i + 1))
        scale = max(np.abs(below[0]).max(), np.abs(below[1]).max())
        for c in (0, 1):
            np.testing.assert_allclose(below[c], above[c], rtol=0, atol=1e-13 * scale)


def test_pw_grid_is_the_point_evaluation_on_the_grid():
    key = 's2d_p0_'
    a = _layer_args(key, 2)
    xs, ys, zs = np.linspace(0, 1, 4), np.linspace(0, 1, 3), np.array([0.0, 0.1])
    G = F.pw_field_grid(a['alphas'], a['betas'], a['sort_order'], a['kz'], a['n'], a['vcd'], a['vcu'],
                        xs, ys, zs, height_norm=a['height_norm'], substrate=False)
    pts = np.array([(x, y, z) for x in xs for y in ys for z in zs])
    P = F.pw_field_points(xyz=pts, **a)
    for c in range(3):
        np.testing.assert_allclose(G[c].ravel(), P[c], rtol=1e-15, atol=0)


def test_bloch_oracle_known_answers():
    """One mode with unit field values: the node values are the mode's
    transverse coefficient (d + u) and E_z's (u - d) / beta, with
    d = v exp(i beta hz), u = v' exp(i beta (h - hz)) (field_value_plane.f:
    104-130); two modes add."""
    nel, M = 3, 2
    sol = np.zeros((nel, M, 13, 3), complex)
    sol[:, 0, :6, :] = 1.0
    sol[1, 1, 2, 0] = 2.0 - 1.0j
    beta = np.array([1.3 + 0.02j, 0.4 + 0.7j])
    v = np.array([0.5 + 0.1j, -0.2j, 0.3, 1.0 + 1.0j])
    h, hz = 0.8, 0.3
    mE = F.bloch_field_plane(sol, beta, v, h, hz)
    d0 = v[0] * np.exp(1j * beta[0] * hz)
    u0 = v[2] * np.exp(1j * beta[0] * (h - hz))
    np.testing.assert_allclose(mE[0, :, 0:2], np.full((6, 2), d0 + u0), rtol=1e-15)
    np.testing.assert_allclose(mE[2, :, 2], np.full(6, (u0 - d0) / beta[0]), rtol=1e-15)
    d1 = v[1] * np.exp(1j * beta[1] * hz)
    u1 = v[3] * np.exp(1j * beta[1] * (h - hz))
    np.testing.assert_allclose(mE[1, 2, 0], d0 + u0 + (2.0 - 1.0j) * (d1 + u1), rtol=1e-15)
    # at the top plane (hz = 0) the down amplitudes enter unpropagated
    mE0 = F.bloch_field_plane(sol, beta, v, h, 0.0)
    np.testing.assert_allclose(mE0[0, 0, 0], v[0] + v[2] * np.exp(1j * beta[0] * h), rtol=1e-15)
    with pytest.raises(ValueError):
        F.bloch_field_plane(sol, beta, v, h, h + 0.1)


def _fake_stacks(name):
    keys = [str(k) for k in GOLD['names'] if str(k).startswith(name + '_')]
    out = []
    for key in keys:
        st = types.SimpleNamespace()
        st.a_list = list(GOLD[key + 'a_list'])
        st.t_list = list(GOLD[key + 't_list'])
        st.r_list = list(GOLD[key + 'r_list'])
        hs = list(GOLD[key + 'heights_nm'])
        st.heights_nm = lambda hs=hs: hs
        out.append((st, float(GOLD[key + 'wl_nm'])))
    return out


@pytest.mark.parametrize('name', ['s2d', 's2c', 's1d'])
def test_text_writer_matches_the_reference_files(name, tmp_path, monkeypatch):
    from emustack_b200.fields import t_r_a_write_files
    monkeypatch.chdir(tmp_path)
    stacks = _fake_stacks(name)
    t_r_a_write_files([s for s, _ in stacks], np.array([w for _, w in stacks]), stack_label=7)
    names = sorted(f for f in os.listdir('.') if f.endswith('.txt'))
    assert names == [str(n) for n in GOLD[name + '_txt_names']]
    for fn, text in zip(names, GOLD[name + '_txt_text']):
        assert open(fn).read() == str(text), fn


def test_zeros_int_str():
    from emustack_b200.fields import zeros_int_str
    assert zeros_int_str(1) == '0001'
    assert zeros_int_str(42) == '0042'
    assert zeros_int_str(12345) == '12345'


def test_save_reference_data_layout(tmp_path, monkeypatch):
    from emustack_b200.fields import save_reference_data
    monkeypatch.chdir(tmp_path)
    rng = np.random.default_rng(0)
    stacks = []
    for _ in range(2):
        lays = [types.SimpleNamespace(**{k: np.asmatrix(rng.normal(size=(4, 4)) + 0j)
                                         for k in ('R12', 'T12', 'R21', 'T21')}, k_z=rng.normal(size=4) + 0j)
                for _ in range(3)]
        stacks.append(types.SimpleNamespace(layers=lays, R_net=np.asmatrix(np.eye(4) + 0j),
                                            T_net=np.asmatrix(2 * np.eye(4) + 0j)))
    path = save_reference_data('case_x', stacks)
    assert path == os.path.join('ref', 'case_x.npz')
    back = np.load(path, allow_pickle=True)['stack_list']
    assert len(back) == 2
    for rs, st in zip(back, stacks):
        np.testing.assert_array_equal(rs['R_net'], st.R_net)
        np.testing.assert_array_equal(rs['T_net'], st.T_net)
        for rl, lay in zip(rs['layers'], st.layers):
            for k in ('R12', 'T12', 'R21', 'T21', 'k_z'):
                np.testing.assert_array_equal(rl[k], getattr(lay, k))
