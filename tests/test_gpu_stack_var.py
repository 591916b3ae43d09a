"""GPU parity of the uneven dense-stack batch (emu_stack_var_batch).

One launch solves stacks of different plane-wave counts, layer counts,
Bloch-mode counts and polarisations, each of which the reference solves with
its own Stack(layers).calc_scat (backend/stack.py:162-426).  Every stack runs
the one-CTA cascade of emu_stack_dense_batch, so results are compared bit for
bit with the uniform batch solved one stack at a time, and with the golden
fixtures (the reference's own outputs) at rtol 1e-9 / atol 1e-10.
"""
import numpy as np
import pytest
import torch

from fixtures import load_points

pytestmark = pytest.mark.gpu

TOL = dict(rtol=1e-9, atol=1e-10)
POLS = ['TE', 'TM', 'un', 'R Circ', 'L Circ']


def _dev_c(x):
    return torch.tensor(np.ascontiguousarray(x, dtype=np.complex128), device='cuda')


def _random_stack(rng, P, Ms, pol, incoming=False):
    """Layers of a random stack: film substrate, films / dense layers with
    the given Bloch-mode counts (0 = film), film superstrate.  Interfaces
    come from the library (film_interface / interface_dense) on random
    J, J_dag; returns per-layer tuples of [1, ...] tensors."""
    from emustack_b200.dense import film_interface, interface_dense
    npw = P // 2
    wln = torch.tensor([rng.uniform(0.8, 2.0)], dtype=torch.float64, device='cuda')
    k0 = 2 * np.pi / float(wln[0])
    kz_air = _dev_c((rng.uniform(0.1, 1.0, npw) + 1j * rng.uniform(0, 0.2, npw)).reshape(1, npw) * k0)
    n_air = _dev_c([1.0])
    layers = []
    for j, M in enumerate([0] + list(Ms) + [0]):
        fin = 0 < j < len(Ms) + 1
        hn = float(rng.uniform(0.05, 0.6))
        if M == 0:
            n = complex(rng.uniform(1.0, 3.0), rng.uniform(0, 0.2)) if j < len(Ms) + 1 else 1.0 + 0j
            kz = _dev_c((rng.uniform(0.1, 1.5, npw) + 1j * rng.uniform(0, 0.3, npw)).reshape(1, npw) * k0)
            R, T = film_interface(kz_air, n_air, kz, _dev_c([n]), wln)
            layers.append((R, T, -R, T, False, torch.cat([kz, kz], 1) if fin else None, hn))
        else:
            J = _dev_c((rng.normal(size=(1, P, M)) + 1j * rng.normal(size=(1, P, M))) / np.sqrt(P))
            Jd = _dev_c((rng.normal(size=(1, M, P)) + 1j * rng.normal(size=(1, M, P))) / np.sqrt(P))
            R12, T12, R21, T21, info = interface_dense(kz_air, n_air, wln, J, Jd)
            assert int(info[0]) == 0
            kz = _dev_c((rng.uniform(0, 2, M) + 1j * rng.uniform(0, 0.1, M)).reshape(1, M) * k0)
            layers.append((R12, T12, R21, T21, True, kz, hn))
    spec = int(rng.integers(0, npw))
    nprop = [int(rng.integers(1, npw + 1)) for _ in range(3)]
    inc = None
    if incoming:
        v = np.zeros(P, complex)
        v[rng.integers(0, P, size=3)] = rng.normal(size=3) + 1j * rng.normal(size=3)
        inc = _dev_c(v.reshape(1, P))
    return dict(layers=layers, P=P, pol=pol, spec=spec, nprop=nprop, inc=inc)


def _uniform(st):
    """The stack alone through emu_stack_dense_batch (one CTA)."""
    from emustack_b200.dense import DenseLayer, DenseStackSolver
    dl = [DenseLayer(R12, T12, R21, T21, d, kz, hn) for R12, T12, R21, T21, d, kz, hn in st['layers']]
    out = DenseStackSolver().solve(dl, st['P'], pol=st['pol'], incoming=st['inc'],
                                   specular=torch.tensor([st['spec']], dtype=torch.int32, device='cuda'),
                                   num_prop=torch.tensor([st['nprop']], dtype=torch.int32, device='cuda'),
                                   mode=1)
    return {k: v.cpu().numpy() for k, v in out.items() if torch.is_tensor(v)}


def _var_stack(st):
    from emustack_b200.dense import VarStack
    lays = [(R12[0], T12[0], R21[0], T21[0], d, None if kz is None else kz[0], hn)
            for R12, T12, R21, T21, d, kz, hn in st['layers']]
    return VarStack(lays, st['P'], pol=st['pol'], incoming=None if st['inc'] is None else st['inc'][0],
                    spec=st['spec'], num_prop=st['nprop'])


def _unpack(out, i, P, L):
    ro, lo = int(out['rnet_off'][i]), int(out['list_off'][i])
    h = out['host']
    return dict(R_net=h['R_net'][ro:ro + P * P].reshape(P, P), T_net=h['T_net'][ro:ro + P * P].reshape(P, P),
                a_list=h['a_list'][lo:lo + L - 1], t_list=h['t_list'][lo:lo + L - 1],
                r_list=h['r_list'][i], flags=int(h['flags'][i]), info=int(h['info'][i]))


def _solve_var(stacks, **kw):
    from emustack_b200.dense import StackVarSolver
    out = StackVarSolver().solve([_var_stack(s) for s in stacks], **kw)
    torch.cuda.synchronize()
    out['host'] = {k: v.cpu().numpy() for k, v in out.items() if torch.is_tensor(v)}
    return out


def test_uneven_batch_matches_uniform_bitwise():
    rng = np.random.default_rng(4)
    stacks = []
    for i in range(24):
        P = int(rng.choice([10, 26, 58, 98]))
        K = int(rng.integers(0, 5))
        Ms = [0 if rng.random() < 0.4 else P + int(rng.integers(-4, 12)) for _ in range(K)]
        stacks.append(_random_stack(rng, P, Ms, POLS[i % 5], incoming=(i % 7 == 3)))
    out = _solve_var(stacks, n_slots=5)
    assert out['n_slots'] == 5
    for i, st in enumerate(stacks):
        u = _uniform(st)
        v = _unpack(out, i, st['P'], len(st['layers']))
        msg = 'stack %d' % i
        np.testing.assert_array_equal(v['R_net'], u['R_net'][0], err_msg=msg)
        np.testing.assert_array_equal(v['T_net'], u['T_net'][0], err_msg=msg)
        np.testing.assert_array_equal(v['a_list'], u['a_list'][0], err_msg=msg)
        np.testing.assert_array_equal(v['t_list'], u['t_list'][0], err_msg=msg)
        np.testing.assert_array_equal(v['r_list'], u['r_list'][0], err_msg=msg)  # nan where no flux
        assert v['flags'] == u['flags'][0] and v['info'] == u['info'][0]


def test_bad_descriptors_are_flagged_and_skipped():
    from emustack_b200 import _lib
    rng = np.random.default_rng(6)
    stacks = [_random_stack(rng, 26, [30, 0], 'TE') for _ in range(6)]
    good = _solve_var(stacks)
    stacks[2]['spec'] = 13                                     # not below P / 2
    R12, T12, R21, T21, d, kz, hn = stacks[4]['layers'][1]
    stacks[4]['layers'][1] = (R12, T12, R21, T21, d, None, hn)  # finite layer without k_z
    bad = _solve_var(stacks)
    for i in range(6):
        g, b = _unpack(good, i, 26, 4), _unpack(bad, i, 26, 4)
        if i in (2, 4):
            assert b['flags'] == _lib.PT_BAD_POINT
        else:
            np.testing.assert_array_equal(b['R_net'], g['R_net'])
            assert b['flags'] == g['flags']


def test_golden_stacks_in_one_launch():
    from emustack_b200.dense import VarStack
    stacks, pts = [], []
    for name in ('case_1', 'case_2', 'case_3', 'case_4', 'case_5', 'synth_config1'):
        gp, _ = load_points(name)
        for pt in gp:
            if pt.get('shears') is not None:
                continue
            lays = []
            nl = len(pt['layers'])
            hs = np.asarray(pt['heights_nm'], float) / float(pt['period'])
            for j, L in enumerate(pt['layers']):
                dense = L['kind'] != 'film'
                mats = []
                for nm in ('R12', 'T12', 'R21', 'T21'):
                    m = np.asarray(L[nm])
                    mats.append(_dev_c(m if dense else np.diag(m)))
                kz = _dev_c(L['k_z']) if 0 < j < nl - 1 else None
                lays.append(tuple(mats) + (dense, kz, hs[j - 1] if 0 < j < nl - 1 else 0.0))
            top, sub = pt['layers'][-1], pt['layers'][0]
            air_np = int(top['num_prop'])   # the superstrate is air in every fixture
            P = len(np.asarray(top['k_z']))
            stacks.append(VarStack(lays, P, pol=pt['pol'], spec=int(top['specular_order']),
                                   num_prop=[air_np, int(top['num_prop']), int(sub['num_prop'])]))
            pts.append(pt)
    assert len(stacks) >= 8
    from emustack_b200.dense import StackVarSolver
    out = StackVarSolver().solve(stacks)
    torch.cuda.synchronize()
    out['host'] = {k: v.cpu().numpy() for k, v in out.items() if torch.is_tensor(v)}
    for i, (st, pt) in enumerate(zip(stacks, pts)):
        v = _unpack(out, i, st.P, len(st.layers))
        np.testing.assert_allclose(v['R_net'], pt['R_net'], **TOL, err_msg='point %d' % i)
        np.testing.assert_allclose(v['T_net'], pt['T_net'], **TOL, err_msg='point %d' % i)
        np.testing.assert_allclose(v['a_list'], np.asarray(pt['a_list'], float), **TOL)
        np.testing.assert_allclose(v['t_list'], np.asarray(pt['t_list'], float), **TOL)
