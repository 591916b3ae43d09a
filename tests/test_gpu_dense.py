"""GPU parity of the dense GSM path: batched complex LU / GEMM, the
film/nanostructure interface (backend/mode_calcs.py:480-515), the cascade
and fluxes (backend/stack.py:162-426) for stacks with nanostructured
layers, through the drop-in objects.  FP64 throughout; held to
rtol 1e-9 / atol 1e-10 against the reference's outputs (product bar: 1e-6
absolute on R, T, A)."""
import numpy as np
import pytest
import torch

from fixtures import load_points, load_raw

pytestmark = pytest.mark.gpu

TOL = dict(rtol=1e-9, atol=1e-10)


def _rand(shape, rng):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize('m,n,k,b', [(1, 1, 1, 1), (5, 7, 3, 2), (64, 64, 64, 1), (70, 130, 65, 3),
                                     (200, 17, 300, 2)])
def test_zgemm_batched(m, n, k, b):
    from emustack_b200.dense import zgemm_batched
    rng = np.random.default_rng(m * 1000 + n)
    A, B, Cc = _rand((b, m, k), rng), _rand((b, k, n), rng), _rand((b, m, n), rng)
    dA, dB, dC = (torch.tensor(x, device='cuda') for x in (A, B, Cc))
    out = zgemm_batched(dA, dB, dC, alpha=0.5 - 2j, beta=1.5 + 0.25j).cpu().numpy()
    np.testing.assert_allclose(out, (0.5 - 2j) * A @ B + (1.5 + 0.25j) * Cc, rtol=1e-12, atol=1e-11)


@pytest.mark.parametrize('n,nrhs,b', [(1, 1, 1), (7, 3, 2), (33, 40, 2), (100, 58, 3), (261, 5, 1)])
def test_zgesv_batched(n, nrhs, b):
    from emustack_b200.dense import zgesv_batched
    rng = np.random.default_rng(n)
    A = _rand((b, n, n), rng) + 3 * np.eye(n)
    Bm = _rand((b, n, nrhs), rng)
    X, ipiv, info = zgesv_batched(torch.tensor(A, device='cuda'), torch.tensor(Bm, device='cuda'))
    assert (info.cpu().numpy() == 0).all()
    np.testing.assert_allclose(X.cpu().numpy(), np.linalg.solve(A, Bm), rtol=1e-10, atol=1e-10)


def test_zgesv_singular_reports_info():
    from emustack_b200.dense import zgesv_batched
    A = np.zeros((1, 4, 4), complex)
    A[0, :3, :3] = np.eye(3)
    _, _, info = zgesv_batched(torch.tensor(A, device='cuda'), torch.ones((1, 4, 1), dtype=torch.complex128,
                                                                          device='cuda'))
    assert int(info[0]) == 4


def test_interface_dense_matches_reference():
    """r_t_mat_tf_ns outputs of the reference at (P, M) = (58, 60), (58, 40), (26, 46)."""
    from emustack_b200.dense import interface_dense
    raw = load_raw('interfaces')
    for q in range(int(raw['n_shapes'])):
        J, Jd = raw['q%d_J' % q], raw['q%d_J_dag' % q]
        kz = raw['q%d_air_kz' % q]
        npw = kz.shape[0]
        dev = 'cuda'
        R12, T12, R21, T21, info = interface_dense(
            torch.tensor(kz.reshape(1, npw), device=dev),
            torch.tensor([1.0 + 0j], dtype=torch.complex128, device=dev),
            torch.tensor([float(raw['q%d_wl_norm' % q])], dtype=torch.float64, device=dev),
            torch.tensor(J[None], device=dev), torch.tensor(Jd[None], device=dev))
        assert int(info[0]) == 0
        for nm, t in (('R12', R12), ('T12', T12), ('R21', R21), ('T21', T21)):
            np.testing.assert_allclose(t[0].cpu().numpy(), raw['q%d_%s' % (q, nm)], rtol=1e-8, atol=1e-9,
                                       err_msg='shape %d %s' % (q, nm))


def _dropin_stack(pt, use_J):
    """Build a drop-in Stack for a golden point: films from n, structured
    layers from J/J_dag (computed interface) or from the stored interface
    matrices injected into the interface memo (as the golden replay does)."""
    from emustack_b200 import objects, materials
    from emustack_b200.mode_calcs import Simmo, _interfaces_i_have_known
    from emustack_b200.stack import Stack
    light = objects.Light(float(pt['wl_nm']), max_order_PWs=int(pt['max_order']),
                          k_parallel=np.asarray(pt['k_pll'], float))
    per, per_y, w1d = float(pt['period']), float(pt['period_y']), bool(pt['world_1d'])
    hs = list(np.asarray(pt['heights_nm'], float))
    nl = len(pt['layers'])
    lays = []
    for i, L in enumerate(pt['layers']):
        h = 'semi_inf' if i in (0, nl - 1) else hs[i - 1]
        if L['kind'] == 'film':
            tf = objects.ThinFilm(per, per_y, height_nm=h, world_1d=w1d,
                                  material=materials.Material(complex(L['n'])), loss=bool(L['loss']))
            lays.append(tf.calc_modes(light))
        else:
            ns = objects.NanoStruct('1D_array' if w1d else '2D_array', per, 100, period_y=per_y,
                                    height_nm=h, world_1d=w1d)
            if use_J and 'J' in L:
                lays.append(ns.calc_modes(light, k_z=L['k_z'], J=L['J'], J_dag=L['J_dag']))
            else:
                sim = Simmo(ns, light)
                sim.k_z = np.asarray(L['k_z'])
                air = sim.air_ref()
                dev = 'cuda'
                _interfaces_i_have_known[(id(air), id(sim))] = {'dev': tuple(
                    torch.tensor(np.ascontiguousarray(L[m]), device=dev).unsqueeze(0)
                    for m in ('R12', 'T12', 'R21', 'T21')) + (True,)}
                lays.append(sim)
    shears = pt.get('shears')
    st = Stack(lays, shears=None if shears is None else [np.asarray(s) for s in shears])
    return st


@pytest.mark.parametrize('name', ['case_1', 'case_2', 'case_3', 'case_4', 'case_5', 'synth_config1',
                                  'synth_shear'])
def test_dense_stack_matches_golden(name):
    pts, raw = load_points(name)
    for p, pt in enumerate(pts):
        st = _dropin_stack(pt, use_J=True)
        st.calc_scat(pol=pt['pol'])
        msg = '%s p%d' % (name, p)
        np.testing.assert_allclose(st.R_net, pt['R_net'], **TOL, err_msg=msg + ' R_net')
        np.testing.assert_allclose(st.T_net, pt['T_net'], **TOL, err_msg=msg + ' T_net')
        np.testing.assert_allclose(np.asarray(st.a_list, float), pt['a_list'], **TOL, err_msg=msg + ' a')
        np.testing.assert_allclose(np.asarray(st.t_list, float), pt['t_list'], **TOL, err_msg=msg + ' t')
        np.testing.assert_allclose(np.asarray(st.r_list, float), pt['r_list'], **TOL, err_msg=msg + ' r')
        for i, L in enumerate(pt['layers']):
            for m in ('R12', 'T12', 'R21', 'T21'):
                np.testing.assert_allclose(getattr(st.layers[i], m), L[m], **TOL, err_msg='%s lay%d %s' % (msg, i, m))
        for a, b in zip(st.vec_coef_down, pt['vec_coef_down']):
            np.testing.assert_allclose(np.ravel(a), b, **TOL)
        for a, b in zip(st.vec_coef_up, pt['vec_coef_up']):
            np.testing.assert_allclose(np.ravel(a), b, **TOL)
        key = 'p%d_stored_R_net' % p
        if key in raw:
            np.testing.assert_allclose(st.R_net, raw[key], rtol=1e-6, atol=1e-6)


def test_save_scat_list_matches_oracle():
    from fixtures import oracle_point
    pts, raw = load_points('synth_config1')
    pt = pts[1]
    st = _dropin_stack(pt, use_J=True)
    st.calc_scat(pol='TE', save_scat_list=True)
    ref = oracle_point(pt)
    assert len(st.rnet_list) == len(ref.rnet_list)
    for a, b in zip(st.rnet_list, ref.rnet_list):
        np.testing.assert_allclose(a, b, **TOL)
    for a, b in zip(st.tnet_list, ref.tnet_list):
        np.testing.assert_allclose(a, b, **TOL)


def test_film_stack_through_dense_path_matches_film_kernel():
    """save_scat_list forces the dense path for an all-film stack; both paths agree."""
    pts, raw = load_points('films10')
    pt = pts[0]
    st = _dropin_stack(pt, use_J=False)
    st.calc_scat(pol=pt['pol'], save_scat_list=True)
    np.testing.assert_allclose(st.R_net, pt['R_net'], **TOL)
    np.testing.assert_allclose(np.asarray(st.a_list, float), pt['a_list'], **TOL)


def _random_dense_stack(rng, B, P, Ms, dense_flags, dev):
    """Substrate film, finite layers (dense with M modes or films), air
    superstrate film: random interface matrices of moderate norm."""
    from emustack_b200.dense import DenseLayer
    c = lambda *s: torch.tensor(_rand(s, rng), device=dev)
    layers = [DenseLayer(*(0.4 * c(B, P) for _ in range(4)), False)]
    for M, dense in zip(Ms, dense_flags):
        kz = torch.tensor(rng.uniform(0, 3, (B, M)) + 1j * rng.uniform(0, 0.3, (B, M)), device=dev)
        if dense:
            R12, T12 = 0.3 * c(B, P, P) / np.sqrt(P), 0.3 * c(B, M, P) / np.sqrt(P)
            R21, T21 = 0.3 * c(B, M, M) / np.sqrt(M), 0.3 * c(B, P, M) / np.sqrt(M)
            layers.append(DenseLayer(R12, T12, R21, T21, True, kz, rng.uniform(0.05, 0.4)))
        else:
            kz = kz[:, :P].contiguous() if M >= P else torch.cat([kz, kz], 1)[:, :P].contiguous()
            layers.append(DenseLayer(*(0.4 * c(B, P) for _ in range(4)), False, kz, rng.uniform(0.05, 0.4)))
    layers.append(DenseLayer(*(0.4 * c(B, P) for _ in range(4)), False))
    return layers


@pytest.mark.parametrize('B,P,Ms,dense,shear,inc', [
    (3, 18, [26, 18], [True, False], False, False),
    (2, 40, [56, 40, 30], [True, False, True], True, False),
    (4, 26, [30], [True], False, True),
    (1, 130, [150, 130], [True, True], True, True),
])
def test_multi_cta_cascade_equals_one_cta_cascade(B, P, Ms, dense, shear, inc):
    """The multi-CTA cascade (each step spread over many CTAs) runs the same
    arithmetic as the one-CTA-per-solve kernel: all outputs are bit-identical."""
    from emustack_b200.dense import DenseStackSolver
    rng = np.random.default_rng(P + len(Ms))
    dev = torch.device('cuda')
    Ms = [M if d else P for M, d in zip(Ms, dense)]
    layers = _random_dense_stack(rng, B, P, Ms, dense, dev)
    npw = P // 2
    spec = torch.tensor(rng.integers(0, npw, B), dtype=torch.int32, device=dev)
    nprop = torch.tensor(rng.integers(1, npw, (B, 3)), dtype=torch.int32, device=dev)
    kw = dict(specular=spec, num_prop=nprop, want_vec_coef=True, save_lists=True)
    if inc:
        kw['incoming'] = torch.tensor(_rand((B, P), rng), device=dev)
    if shear:
        kw['shears'] = [rng.uniform(-0.3, 0.3, 2) for _ in range(len(layers))]
        kw['air_alphas'] = torch.tensor(rng.uniform(-3, 3, (B, npw)), device=dev)
        kw['air_betas'] = torch.tensor(rng.uniform(-3, 3, (B, npw)), device=dev)
    outs = []
    for mode in (1, 2):
        o = DenseStackSolver(dev).solve(layers, P, pol='TM', mode=mode, **kw)
        torch.cuda.synchronize()
        outs.append({k: v.cpu() for k, v in o.items() if isinstance(v, torch.Tensor)})
    assert int(outs[0]['info'].abs().sum()) == 0
    for k in outs[0]:
        assert torch.equal(outs[0][k], outs[1][k]), k


def test_multi_cta_cascade_reports_singular_solve():
    """A gap solve with an exactly singular matrix reports the same info code
    in both cascades (first zero pivot, continuing as LAPACK does)."""
    from emustack_b200.dense import DenseLayer, DenseStackSolver
    dev = torch.device('cuda')
    B, P = 2, 6
    one = torch.ones((B, P), dtype=torch.complex128, device=dev)
    z = torch.zeros((B, P), dtype=torch.complex128, device=dev)
    # substrate reflects fully, superstrate R12 = 1: I - R12 rnet = 0
    layers = [DenseLayer(one, one, -one, one, False), DenseLayer(one, one, -one, one, False)]
    infos = []
    for mode in (1, 2):
        o = DenseStackSolver(dev).solve(layers, P, calc_fluxes=False, mode=mode)
        infos.append(o['info'].cpu().numpy())
    assert (infos[0] != 0).all() and np.array_equal(infos[0], infos[1])


@pytest.mark.parametrize('B,P,M', [(2, 26, 30), (1, 130, 150), (3, 58, 40)])
def test_multi_cta_interface_equals_one_cta_interface(B, P, M):
    """Film/nanostructure interfaces through the multi-CTA path (forced with
    emu_set_dense_mode) equal the one-CTA kernel: same LU, solves and GEMMs;
    the film impedances are formed in a different kernel, where the compiler
    may contract multiply-adds differently; those last-bit differences pass
    through the M x M solve, so agreement is held to 1e-10 of max |entry|."""
    from emustack_b200 import _lib
    from emustack_b200.dense import interface_dense
    rng = np.random.default_rng(P * M)
    dev = torch.device('cuda')
    npw = P // 2
    kz = torch.tensor(rng.uniform(0.1, 3, (B, npw)) + 1j * rng.uniform(0, 0.5, (B, npw)), device=dev)
    n = torch.tensor(rng.uniform(1.0, 2.0, B) + 0j, device=dev)
    wln = torch.tensor(rng.uniform(0.6, 1.5, B), device=dev)
    J = torch.tensor(_rand((B, P, M), rng) / np.sqrt(P), device=dev)
    Jd = torch.tensor(_rand((B, M, P), rng) / np.sqrt(P), device=dev)
    L = _lib.lib()
    outs = []
    try:
        for mode in (1, 2):
            L.emu_set_dense_mode(mode)
            o = interface_dense(kz, n, wln, J, Jd)
            torch.cuda.synchronize()
            outs.append([t.cpu() for t in o])
    finally:
        L.emu_set_dense_mode(0)
    for a, b in zip(*outs):
        a, b = a.numpy(), b.numpy()
        assert np.abs(a - b).max() <= 1e-10 * max(np.abs(a).max(), 1.0)


class _PlainFilm(object):
    """A film layer that is not an emustack_b200 class: the attributes and
    methods the reference's Anallo exposes (backend/mode_calcs.py:99-250)."""

    def __init__(self, src, air=None):
        for nm in ('structure', 'light', 'k_z', 'specular_order', 'num_prop_pw_per_pol',
                   'sort_order', 'alphas', 'betas', 'is_air_ref', 'max_order_PWs'):
            setattr(self, nm, getattr(src, nm))
        self._n = src.n()
        self._wl_norm = src.wl_norm()
        self._air = air if air is not None else self

    def n(self):
        return self._n

    def k(self):
        return np.complex128(2 * np.pi * self.n() / self.wl_norm())

    def wl_norm(self):
        return self._wl_norm

    def air_ref(self):
        return self._air

    def Z(self):
        npw = len(self.k_z) // 2
        k_on_kz = self.k() / self.k_z[:npw]
        return np.concatenate((k_on_kz / self.n(), 1 / (self.n() * k_on_kz)))

    def specular_incidence(self, pol='TE'):
        raise AssertionError('not read by the GSM stage')


class _PlainSimmo(object):
    """A nanostructured layer that is not an emustack_b200 class: k_z, J,
    J_dag and the structure/light, as the reference's Simmo holds them."""

    def __init__(self, src, air):
        for nm in ('structure', 'light', 'k_z', 'J', 'J_dag'):
            setattr(self, nm, getattr(src, nm))
        self._air = air

    def air_ref(self):
        return self._air


@pytest.mark.parametrize('name', ['synth_config1', 'films10'])
def test_dropin_accepts_plain_layer_objects(name):
    """Stack dispatches on the layer interface (Z / specular_incidence for
    films, J / J_dag for nanostructured layers), not on this package's
    classes: stand-in objects built like the reference's Anallo / Simmo give
    the same R_net, T_net and a/t/r lists."""
    from emustack_b200.mode_calcs import is_film
    from emustack_b200.stack import Stack
    pts, _ = load_points(name)
    pt = pts[0]
    st = _dropin_stack(pt, use_J=True)
    st.calc_scat(pol=pt['pol'])
    air = _PlainFilm(st.layers[-1].air_ref())
    plain = [_PlainFilm(l, air) if is_film(l) else _PlainSimmo(l, air) for l in st.layers]
    assert not any(type(l).__module__.startswith('emustack_b200') for l in plain)
    st2 = Stack(plain, shears=st.shears)
    st2.calc_scat(pol=pt['pol'])
    np.testing.assert_allclose(st2.R_net, st.R_net, rtol=0, atol=0)
    np.testing.assert_allclose(st2.T_net, st.T_net, rtol=0, atol=0)
    for k in ('a_list', 't_list', 'r_list'):
        np.testing.assert_allclose(np.asarray(getattr(st2, k), float), np.asarray(getattr(st, k), float),
                                   rtol=1e-12, atol=1e-14, err_msg=k)
    np.testing.assert_allclose(st2.R_net, pt['R_net'], **TOL)
