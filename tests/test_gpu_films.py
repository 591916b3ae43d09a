"""GPU parity of the fused all-film GSM kernel (emu_film_stack_batch).

Reference behaviour: backend/stack.py:162-426 with every layer an Anallo
(backend/mode_calcs.py:99-250, 451-477).  Tolerance: the GPU path computes
in FP64 like the reference, so results are held to rtol 1e-9 / atol 1e-10
(the product bar is 1e-6 absolute on R, T, A).
"""
import numpy as np
import pytest
import torch

from fixtures import film_inputs, load_points

pytestmark = pytest.mark.gpu

TOL = dict(rtol=1e-9, atol=1e-10)


def _solve_point(fi, want=('kz', 'layer_rt', 'vec_coef', 'fluxes', 'sort_order', 'specular', 'num_prop')):
    from emustack_b200.films import FilmStackSolver
    L = len(fi['n'])
    s = FilmStackSolver(L, fi['max_order'], fi['period'], fi['period_y'], fi['world_1d'])
    dev = s.device
    wl = torch.tensor([fi['wl']], dtype=torch.float64, device=dev)
    kp = torch.tensor(fi['k_pll'].reshape(1, 2), device=dev)
    n = torch.tensor(fi['n'].reshape(1, L), dtype=torch.complex128, device=dev)
    hs = torch.tensor(fi['heights'], device=dev)
    inc = None if fi['incoming'] is None else torch.tensor(fi['incoming'].reshape(1, -1), device=dev)
    sh = None if fi['shears'] is None else torch.tensor(fi['shears'], device=dev)
    out = s.solve(wl, kp, n, hs, pol=fi['pol'], incoming=inc, shears=sh, want=want)
    torch.cuda.synchronize()
    return s, {k: v.cpu().numpy() for k, v in out.items()}


@pytest.mark.parametrize('name', ['case_0', 'films10', 'edge_cases'])
def test_film_kernel_matches_golden(name):
    pts, raw = load_points(name)
    for p, pt in enumerate(pts):
        fi = film_inputs(pt)
        s, o = _solve_point(fi)
        L = len(fi['n'])
        msg = '%s p%d' % (name, p)
        np.testing.assert_allclose(np.diag(o['R_net'][0]), pt['R_net'], **TOL, err_msg=msg + ' R_net')
        np.testing.assert_allclose(np.diag(o['T_net'][0]), pt['T_net'], **TOL, err_msg=msg + ' T_net')
        if o['flags'][0] & 4:   # no propagating orders in the substrate: zeros(L-2)
            assert np.all(pt['a_list'] == 0)
        else:
            np.testing.assert_allclose(o['a_list'][0], pt['a_list'], **TOL, err_msg=msg + ' a')
            np.testing.assert_allclose(o['t_list'][0], pt['t_list'], **TOL, err_msg=msg + ' t')
            np.testing.assert_allclose(o['r_list'][0:1], pt['r_list'], **TOL, err_msg=msg + ' r')
        for i, lay in enumerate(pt['layers']):
            np.testing.assert_allclose(o['kz'][0, i], lay['k_z'][:s.npw], **TOL, err_msg=msg + ' kz')
            np.testing.assert_allclose(np.diag(o['layer_rt'][0, i, 0]), lay['R12'], **TOL)
            np.testing.assert_allclose(np.diag(o['layer_rt'][0, i, 1]), lay['T12'], **TOL)
            assert int(o['num_prop'][0, i]) == int(lay['num_prop'])
            assert int(o['specular'][0]) == int(lay['specular_order'])
        for lv in range(L):
            np.testing.assert_allclose(o['vec_coef_down'][0, lv], pt['vec_coef_down'][lv], **TOL)
        for lv in range(L - 1):
            np.testing.assert_allclose(o['vec_coef_up'][0, lv], pt['vec_coef_up'][lv], **TOL)


def test_wood_anomaly_flag():
    pts, raw = load_points('edge_cases')
    fi = film_inputs(pts[2])
    s, o = _solve_point(fi)
    assert o['flags'][0] & 1
    np.testing.assert_allclose(o['kz'][0, -1], raw['p2_air_kz'][:s.npw], **TOL)


def test_stack_api_case0():
    """tests/test_case_0_thin_film_multistack.py, through the drop-in objects."""
    from emustack_b200 import objects, materials
    from emustack_b200.stack import Stack
    pts, raw = load_points('case_0')
    for p, pt in enumerate(pts):
        ns = [complex(L['n']) for L in pt['layers']]
        loss = [bool(L['loss']) for L in pt['layers']]
        light = objects.Light(float(pt['wl_nm']), max_order_PWs=1, theta=0.0, phi=0.0)
        hs = [None] + list(pt['heights_nm']) + [None]
        films = [objects.ThinFilm(period=1, height_nm=('semi_inf' if h is None else h),
                                  material=materials.Material(n), loss=lo)
                 for n, h, lo in zip(ns, hs, loss)]
        st = Stack([f.calc_modes(light) for f in films])
        st.calc_scat(pol='TM')
        np.testing.assert_allclose(st.R_net, raw['p%d_stored_R_net' % p], rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(st.T_net, raw['p%d_stored_T_net' % p], rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(st.R_net, pt['R_net'], **TOL)
        np.testing.assert_allclose(st.a_list, pt['a_list'], **TOL)
        for i, lay in enumerate(st.layers):
            np.testing.assert_allclose(lay.k_z, pt['layers'][i]['k_z'], **TOL)
            np.testing.assert_allclose(lay.R12, pt['layers'][i]['R12'], **TOL)
            np.testing.assert_allclose(lay.T21, pt['layers'][i]['T21'], **TOL)


def _config2_stack(seed=0, L=10):
    rng = np.random.default_rng(seed)
    h = rng.uniform(20, 300, L)
    n = rng.uniform(1.3, 4.0, L) + 1j * rng.uniform(0, 0.5, L)
    return h, np.concatenate([[1.46 + 0j], n, [1.0 + 0j]])


def _points(B, seed=1):
    from oracle.gsm_oracle import k_parallel_from_angles
    rng = np.random.default_rng(seed)
    wl = rng.uniform(350, 1100, B)
    th = rng.uniform(0, 60, B)
    ph = rng.uniform(0, 90, B)
    kp = np.array([k_parallel_from_angles(w, t, f) for w, t, f in zip(wl, th, ph)])
    return wl, kp


@pytest.mark.parametrize('pol', ['TE', 'TM', 'R Circ'])
def test_film_batch_vs_oracle(pol):
    """Batched thin-film workload shape (10 films, period 500, max order 5)."""
    from oracle import gsm_oracle as O
    from emustack_b200.films import FilmStackSolver
    h, nl = _config2_stack()
    B = 24
    wl, kp = _points(B)
    s = FilmStackSolver(len(nl), 5, 500.0)
    dev = s.device
    out = s.solve(torch.tensor(wl, device=dev), torch.tensor(kp, device=dev),
                  torch.tensor(np.tile(nl, (B, 1)), device=dev), torch.tensor(h, device=dev), pol=pol)
    o = {k: v.cpu().numpy() for k, v in out.items()}
    for b in range(B):
        r = O.film_stack_point(nl, h, wl[b], kp[b], 500.0, max_order=5, pol=pol)
        np.testing.assert_allclose(o['R_net'][b], np.diag(r.R_net), **TOL)
        np.testing.assert_allclose(o['T_net'][b], np.diag(r.T_net), **TOL)
        np.testing.assert_allclose(o['a_list'][b], np.asarray(r.a_list, float), rtol=1e-9, atol=1e-9)
        np.testing.assert_allclose(o['t_list'][b], np.asarray(r.t_list, float), rtol=1e-9, atol=1e-9)
        np.testing.assert_allclose(o['r_list'][b], float(r.r_list[0]), rtol=1e-9, atol=1e-9)


def test_film_shears_vs_oracle():
    from oracle import gsm_oracle as O
    from emustack_b200.films import FilmStackSolver
    h, nl = _config2_stack(seed=3, L=4)
    shears = np.array([[0.0, 0.0], [0.1, 0.25], [0.3, 0.05], [0.2, 0.2], [0.45, 0.1], [0.05, 0.3]])
    B = 6
    wl, kp = _points(B, seed=4)
    s = FilmStackSolver(len(nl), 3, 500.0)
    dev = s.device
    out = s.solve(torch.tensor(wl, device=dev), torch.tensor(kp, device=dev),
                  torch.tensor(np.tile(nl, (B, 1)), device=dev), torch.tensor(h, device=dev),
                  pol='un', shears=torch.tensor(shears, device=dev))
    o = {k: v.cpu().numpy() for k, v in out.items()}
    for b in range(B):
        r = O.film_stack_point(nl, h, wl[b], kp[b], 500.0, max_order=3, pol='un', shears=list(shears))
        np.testing.assert_allclose(o['R_net'][b], np.diag(r.R_net), **TOL)
        np.testing.assert_allclose(o['T_net'][b], np.diag(r.T_net), **TOL)
        np.testing.assert_allclose(o['a_list'][b], np.asarray(r.a_list, float), rtol=1e-9, atol=1e-9)


def test_full_size_batch_properties():
    """Full batched workload (2048 wavelengths x 16 angles): lossless stacks
    conserve energy, every point is finite, and results do not depend on the
    batch a point is solved in (bitwise)."""
    from emustack_b200.films import FilmStackSolver
    h, nl = _config2_stack()
    B = 2048 * 16
    wl, kp = _points(B, seed=7)
    s = FilmStackSolver(len(nl), 5, 500.0)
    dev = s.device
    n_lossless = np.tile(nl.real + 0j, (B, 1))
    out = s.solve(torch.tensor(wl, device=dev), torch.tensor(kp, device=dev),
                  torch.tensor(n_lossless, device=dev), torch.tensor(h, device=dev), pol='TE')
    a = out['a_list'].cpu().numpy()
    t = out['t_list'].cpu().numpy()
    r = out['r_list'].cpu().numpy()
    assert np.all(np.isfinite(a)) and np.all(np.isfinite(t)) and np.all(np.isfinite(r))
    np.testing.assert_allclose(a[:, -1], 0.0, atol=1e-9)
    np.testing.assert_allclose(r + t[:, -1], 1.0, atol=1e-9)
    # lossy: 0 <= A, R, T and A + R + T = 1
    n_lossy = torch.tensor(np.tile(nl, (B, 1)), device=dev)
    out = s.solve(torch.tensor(wl, device=dev), torch.tensor(kp, device=dev), n_lossy,
                  torch.tensor(h, device=dev), pol='TE')
    full = {k: v.clone() for k, v in out.items()}
    a = full['a_list'].cpu().numpy()
    t = full['t_list'].cpu().numpy()
    r = full['r_list'].cpu().numpy()
    np.testing.assert_allclose(a[:, -1] + r + t[:, -1], 1.0, atol=1e-9)
    sub = np.arange(5, B, 997)
    s2 = FilmStackSolver(len(nl), 5, 500.0)
    o2 = s2.solve(torch.tensor(wl[sub], device=dev), torch.tensor(kp[sub], device=dev),
                  n_lossy[sub].contiguous(), torch.tensor(h, device=dev), pol='TE')
    assert torch.equal(o2['R_net'], full['R_net'][sub])
    assert torch.equal(o2['a_list'], full['a_list'][sub])


@pytest.mark.parametrize('pol', ['un', 'incoming'])
def test_launch_variants_agree(pol):
    """Every launch variant of the film kernel gives the same result: the
    per-order quantities (R_net, T_net, k_z, interface r/t, mode vectors)
    bit for bit, the flux sums (a/t/r lists, fluxes) to rounding, since the
    teams add them up with shared-memory atomics in no fixed order."""
    from emustack_b200 import _lib
    from emustack_b200.films import FilmStackSolver
    h, nl = _config2_stack(seed=5, L=6)
    B = 40
    wl, kp = _points(B, seed=9)
    s = FilmStackSolver(len(nl), 4, 500.0)
    dev = s.device
    inc = None
    if pol == 'incoming':
        rng = np.random.default_rng(2)
        inc = rng.normal(size=(B, 2 * s.npw)) + 1j * rng.normal(size=(B, 2 * s.npw))
        inc[:, rng.random(2 * s.npw) < 0.6] = 0
        inc = torch.tensor(inc, device=dev)
    shears = torch.tensor(np.linspace(0, 0.4, 2 * len(nl)).reshape(len(nl), 2), device=dev)
    want = ('kz', 'layer_rt', 'vec_coef', 'fluxes', 'num_prop')
    args = (torch.tensor(wl, device=dev), torch.tensor(kp, device=dev),
            torch.tensor(np.tile(nl, (B, 1)), device=dev), torch.tensor(h, device=dev))
    res = {}
    for v in _lib.FILM_VARIANTS:
        out = s.solve(*args, pol='un' if inc is None else 'incoming', incoming=inc, shears=shears,
                      want=want, variant=v)
        res[v] = {k: t.cpu().numpy().copy() for k, t in out.items()}
    exact = ('R_net', 'T_net', 'kz', 'layer_rt', 'vec_coef_down', 'vec_coef_up', 'flags', 'num_prop')
    for v in _lib.FILM_VARIANTS[1:]:
        for k, x in res[v].items():
            if k in exact:
                np.testing.assert_array_equal(x, res[0][k], err_msg='variant %d %s' % (v, k))
            else:
                np.testing.assert_allclose(x, res[0][k], rtol=1e-12, atol=1e-14,
                                           err_msg='variant %d %s' % (v, k))


@pytest.mark.parametrize('per_point_heights', [False, True])
def test_host_pipeline_matches_device_solve(per_point_heights):
    """FilmHostPipeline (host inputs, pieces on two streams, pinned host
    outputs) gives the device solver's results bit for bit, also when the
    batch is not a multiple of the piece size."""
    from emustack_b200.films import FilmHostPipeline, FilmStackSolver
    h, nl = _config2_stack(seed=2)
    B = 1000
    wl, kp = _points(B, seed=5)
    n = np.tile(nl, (B, 1))
    hs = np.tile(h, (B, 1)) * np.linspace(0.5, 1.5, B)[:, None] if per_point_heights else h
    pipe = FilmHostPipeline(len(nl), 5, 500.0, chunk=300)
    host = [torch.tensor(a).pin_memory() for a in (wl, kp, n, hs)]
    out = pipe.solve(*host, pol='un')
    torch.cuda.synchronize()
    s = FilmStackSolver(len(nl), 5, 500.0)
    dev = s.device
    ref = s.solve(*[t.to(dev) for t in host], pol='un')
    for k in FilmHostPipeline.OUT:
        np.testing.assert_array_equal(out[k].numpy(), ref[k].cpu().numpy(), err_msg=k)


def test_host_pipeline_spectra_only():
    """FilmHostPipeline(outputs=SPECTRA) brings back only the a/t/r lists and
    flags, equal to the full device solve's."""
    from emustack_b200.films import FilmHostPipeline, FilmStackSolver
    h, nl = _config2_stack(seed=3)
    B = 700
    wl, kp = _points(B, seed=6)
    n = np.tile(nl, (B, 1))
    pipe = FilmHostPipeline(len(nl), 5, 500.0, chunk=256, outputs=FilmHostPipeline.SPECTRA)
    host = [torch.tensor(a).pin_memory() for a in (wl, kp, n, h)]
    out = pipe.solve(*host, pol='TM')
    torch.cuda.synchronize()
    assert set(out) == set(FilmHostPipeline.SPECTRA)
    s = FilmStackSolver(len(nl), 5, 500.0)
    ref = s.solve(*[t.to(s.device) for t in host], pol='TM')
    for k in FilmHostPipeline.SPECTRA:
        np.testing.assert_array_equal(out[k].numpy(), ref[k].cpu().numpy(), err_msg=k)
    with pytest.raises(ValueError):
        FilmHostPipeline(len(nl), 5, 500.0, outputs=('R_net', 'nonsense'))
