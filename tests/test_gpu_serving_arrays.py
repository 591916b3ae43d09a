"""GPU parity of array-stack requests in the continuous-batching server.

An ArrayRequest is one spectral point of a stack with nanostructured layers,
solved by the reference with Stack(layers).calc_scat(pol)
(backend/stack.py:162-426) after r_t_mat of each layer
(backend/mode_calcs.py:416-515).  Checked against the golden fixtures (the
reference's own outputs), against the CPU oracle, alone against in a mix of
shapes and film requests, and through the device cache of layer interfaces
(hits, evictions).  Tolerance: FP64 throughout, rtol 1e-9 / atol 1e-10
against the fixtures and the oracle; a request alone and in the mix runs the
same per-point code, held to rtol 1e-12.
"""
import numpy as np
import pytest

from fixtures import load_points

pytestmark = pytest.mark.gpu

TOL = dict(rtol=1e-9, atol=1e-10)


def _film_n(L):
    v = complex(L['n'])
    return v if bool(L['loss']) else complex(v.real, 0.0)


def _golden_request(pt, use_J):
    from emustack_b200.array_serving import ArrayLayer, ArrayRequest
    layers = []
    for L in pt['layers']:
        if L['kind'] == 'film':
            layers.append(_film_n(L))
        elif use_J and 'J' in L:
            layers.append(ArrayLayer(L['k_z'], J=L['J'], J_dag=L['J_dag']))
        else:
            layers.append(ArrayLayer(L['k_z'], rt=(L['R12'], L['T12'], L['R21'], L['T21'])))
    return ArrayRequest(layers, pt['heights_nm'], float(pt['wl_nm']), pt['k_pll'], float(pt['period']),
                        int(pt['max_order']), pol=pt['pol'], period_y=float(pt['period_y']),
                        world_1d=bool(pt['world_1d']))


def _golden_cases():
    out = []
    for name in ('case_1', 'case_2', 'case_3', 'case_4', 'case_5', 'synth_config1'):
        pts, _ = load_points(name)
        for i, pt in enumerate(pts):
            if pt.get('shears') is not None or pt.get('incoming') is not None:
                continue
            out.append(('%s p%d' % (name, i), pt))
    return out


# uneven_max_dim 0: every array request grouped by shape; 1024: every one in
# the one-launch uneven batch
@pytest.mark.parametrize('use_J,uneven', [(False, 0), (True, 0), (False, 1024), (True, 1024)])
def test_golden_array_requests(use_J, uneven):
    from emustack_b200.serving import GsmServer
    cases = _golden_cases()
    assert len(cases) >= 8
    with GsmServer(hbm_budget_bytes=8 << 30, smatrix_cache_bytes=1 << 30, uneven_max_dim=uneven) as srv:
        futs = [(msg, pt, srv.submit(_golden_request(pt, use_J))) for msg, pt in cases]
        for msg, pt, f in futs:
            r = f.result(timeout=300)
            np.testing.assert_allclose(r['R_net'], pt['R_net'], **TOL, err_msg=msg + ' R_net')
            np.testing.assert_allclose(r['T_net'], pt['T_net'], **TOL, err_msg=msg + ' T_net')
            np.testing.assert_allclose(r['a_list'], np.asarray(pt['a_list'], float), **TOL, err_msg=msg)
            np.testing.assert_allclose(r['t_list'], np.asarray(pt['t_list'], float), **TOL, err_msg=msg)
            np.testing.assert_allclose(r['r_list'], float(np.asarray(pt['r_list']).ravel()[0]), **TOL)
    assert srv.error is None


def _random_layer(rng, P, M, wl_nm, period, max_order):
    """A synthetic array layer at one spectral point: J, J_dag complex
    N(0, 1)/sqrt(P), Bloch k_z with Re U(0, 2 k0), Im U(0, 0.1 k0)."""
    from emustack_b200.array_serving import ArrayLayer
    k0 = 2 * np.pi / (wl_nm / period)
    J = (rng.normal(size=(P, M)) + 1j * rng.normal(size=(P, M))) / np.sqrt(P)
    Jd = (rng.normal(size=(M, P)) + 1j * rng.normal(size=(M, P))) / np.sqrt(P)
    kz = rng.uniform(0, 2, M) * k0 + 1j * rng.uniform(0, 0.1, M) * k0
    return ArrayLayer(kz, J=J, J_dag=Jd), (kz, J, Jd)


def _oracle(req, raw):
    """The oracle's solve of one array request; raw maps an ArrayLayer's
    key to its (k_z, J, J_dag)."""
    from oracle import gsm_oracle as O
    from emustack_b200.array_serving import ArrayLayer
    air = O.make_air_ref(req.wl_nm, req.k_pll, req.period, req.period_y, req.max_order, req.world_1d)
    layers = []
    L = len(req.layers)
    for i, ly in enumerate(req.layers):
        h = None if i in (0, L - 1) else float(req.heights[i - 1])
        if isinstance(ly, ArrayLayer):
            kz, J, Jd = raw[ly.key]
            layers.append(O.OracleLayer('struct', kz, h, J=np.asmatrix(J), J_dag=np.asmatrix(Jd)))
        else:
            layers.append(O.film_layer(ly, req.wl_nm, req.k_pll, req.period, air, h, req.period_y,
                                       req.max_order, req.world_1d))
    return O.calc_scat(layers, air, req.period, pol=req.pol, heights_nm=list(req.heights))


def _mixed_workload(rng, n_array, n_film):
    from emustack_b200.array_serving import ArrayRequest
    from emustack_b200.films import grating_orders
    from emustack_b200.serving import FilmRequest
    from oracle.gsm_oracle import k_parallel_from_angles
    period = 500.0
    pool, raw = [], {}
    # a pool of layers at a few spectral points, two order sets
    points = []
    for mo in (2, 3):
        P = 2 * len(grating_orders(mo, period)[0])
        for _ in range(3):
            wl = float(rng.uniform(450, 1000))
            kp = k_parallel_from_angles(wl, float(rng.uniform(0, 30)), float(rng.uniform(0, 90)))
            lays = []
            for M in (P + 4, P + 10):
                ly, data = _random_layer(rng, P, M, wl, period, mo)
                raw[ly.key] = data
                lays.append(ly)
            points.append((mo, wl, kp, lays))
    reqs = []
    pols = ['TE', 'TM', 'un', 'R Circ']
    for i in range(n_array):
        mo, wl, kp, lays = points[int(rng.integers(len(points)))]
        K = int(rng.integers(1, 4))
        mid = []
        for k in range(K):
            mid.append(lays[int(rng.integers(len(lays)))] if rng.random() < 0.7
                       else complex(rng.uniform(1.3, 3.5), rng.uniform(0, 0.2)))
        layers = [complex(rng.uniform(1.3, 2.0), 0.0)] + mid + [1.0 + 0j]
        hs = rng.uniform(50, 300, K)
        reqs.append(ArrayRequest(layers, hs, wl, kp, period, mo, pol=pols[i % 4]))
    for i in range(n_film):
        L = int(rng.integers(3, 8))
        wl = float(rng.uniform(400, 1000))
        kp = k_parallel_from_angles(wl, float(rng.uniform(0, 40)), 0.0)
        n = np.concatenate([[1.46 + 0j], rng.uniform(1.3, 3.5, L - 2) + 1j * rng.uniform(0, 0.3, L - 2),
                            [1.0 + 0j]])
        reqs.append(FilmRequest(n, rng.uniform(20, 300, L - 2), wl, kp, period, 3, pol='TE'))
    order = rng.permutation(len(reqs))
    return [reqs[i] for i in order], raw


@pytest.mark.parametrize('uneven', [0, 1024])
def test_array_requests_alone_and_in_the_mix(uneven):
    """In the mix: shapes and film requests together (uneven batches or
    shape groups); alone: a fresh server, grouped path.  Both paths run the
    same per-stack arithmetic."""
    from emustack_b200.array_serving import ArrayRequest
    from emustack_b200.serving import GsmServer
    rng = np.random.default_rng(11)
    reqs, raw = _mixed_workload(rng, 60, 60)
    with GsmServer(hbm_budget_bytes=8 << 30, smatrix_cache_bytes=1 << 30, n_streams=3,
                   uneven_max_dim=uneven) as srv:
        futs = [srv.submit(r) for r in reqs]
        mix = [f.result(timeout=300) for f in futs]
        st = srv.stats()
    assert srv.error is None
    c = st['smatrix_cache']
    assert c['misses'] <= 12          # every pool layer's interface computed at most once
    arrays = [i for i, r in enumerate(reqs) if isinstance(r, ArrayRequest)]
    for k, i in enumerate(arrays[:12]):
        r = reqs[i]
        with GsmServer(hbm_budget_bytes=4 << 30, smatrix_cache_bytes=1 << 30, uneven_max_dim=0) as one:
            alone = one.submit(r).result(timeout=300)
        for key in ('R_net', 'T_net', 'a_list', 't_list'):
            np.testing.assert_allclose(mix[i][key], alone[key], rtol=1e-12, atol=1e-14,
                                       err_msg='request %d %s' % (i, key))
        assert mix[i]['flags'] == alone['flags']
        if k < 6:
            o = _oracle(r, raw)
            np.testing.assert_allclose(mix[i]['R_net'], o.R_net, **TOL, err_msg='request %d' % i)
            np.testing.assert_allclose(mix[i]['T_net'], o.T_net, **TOL, err_msg='request %d' % i)
            np.testing.assert_allclose(mix[i]['a_list'], np.asarray(o.a_list, float), **TOL)
            np.testing.assert_allclose(mix[i]['t_list'], np.asarray(o.t_list, float), **TOL)


def test_thickness_sweep_reuses_the_cached_interface():
    """A sweep over the height of one array layer computes its interface
    once; every point matches the oracle."""
    from emustack_b200.array_serving import ArrayRequest
    from emustack_b200.serving import GsmServer
    from oracle.gsm_oracle import k_parallel_from_angles
    rng = np.random.default_rng(5)
    wl, period, mo = 640.0, 600.0, 3
    kp = k_parallel_from_angles(wl, 12.0, 30.0)
    from emustack_b200.films import grating_orders
    P = 2 * len(grating_orders(mo, period)[0])
    ly, data = _random_layer(rng, P, P + 6, wl, period, mo)
    raw = {ly.key: data}
    hs = np.linspace(20.0, 400.0, 40)
    reqs = [ArrayRequest([1.46 + 0j, ly, 1.0 + 0j], [h], wl, kp, period, mo, pol='TM') for h in hs]
    with GsmServer(hbm_budget_bytes=4 << 30, smatrix_cache_bytes=1 << 30) as srv:
        first = srv.submit(reqs[0]).result(timeout=300)
        futs = [srv.submit(r) for r in reqs[1:]]
        res = [first] + [f.result(timeout=300) for f in futs]
        c = srv.stats()['smatrix_cache']
    assert c['misses'] == 1 and c['hits'] >= 1 and c['entries'] == 1
    for i in (0, 7, 19, 39):
        o = _oracle(reqs[i], raw)
        np.testing.assert_allclose(res[i]['R_net'], o.R_net, **TOL)
        np.testing.assert_allclose(res[i]['a_list'], np.asarray(o.a_list, float), **TOL)
    # the height changes the result (the cached interface is not the answer)
    assert np.abs(res[0]['R_net'] - res[-1]['R_net']).max() > 1e-3


def test_cache_eviction_keeps_results():
    """With room for two layers only, the server evicts and recomputes
    interfaces; results are those of a server that keeps every layer."""
    from emustack_b200.serving import GsmServer
    rng = np.random.default_rng(8)
    reqs, _ = _mixed_workload(rng, 40, 0)
    from emustack_b200.array_serving import ArrayRequest
    arrays = [r for r in reqs if isinstance(r, ArrayRequest)]
    big = max(ly.smatrix_bytes() for r in arrays for ly in r.layers if not isinstance(ly, complex))
    outs = []
    for cap in (1 << 30, 2 * big):
        with GsmServer(hbm_budget_bytes=4 << 30, smatrix_cache_bytes=cap, n_streams=2) as srv:
            outs.append([f.result(timeout=300) for f in [srv.submit(r) for r in arrays]])
            outs[-1].append(srv.stats()['smatrix_cache'])
    assert outs[1][-1]['evictions'] > 0 and outs[0][-1]['evictions'] == 0
    for a, b in zip(outs[0][:-1], outs[1][:-1]):
        np.testing.assert_allclose(a['R_net'], b['R_net'], rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(a['a_list'], b['a_list'], rtol=1e-12, atol=1e-14)
