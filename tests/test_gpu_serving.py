"""Continuous batching (emustack_b200.serving): requests arriving while
batches run are admitted into later launches, every result equals the same
point solved alone (bitwise) and the oracle (1e-9).  The default 'mixed'
mode puts requests of any shape into one uneven-batch launch; 'grouped'
batches one shape per launch of the uniform kernel."""
import threading
import time

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _requests(n_req, seed=0):
    from emustack_b200.serving import FilmRequest
    from oracle.gsm_oracle import k_parallel_from_angles
    rng = np.random.default_rng(seed)
    stacks = []
    for L in (5, 8):
        n = np.concatenate([[1.46 + 0j], rng.uniform(1.3, 4.0, L - 2) + 1j * rng.uniform(0, 0.5, L - 2), [1.0 + 0j]])
        stacks.append((n, rng.uniform(20, 300, L - 2)))
    reqs = []
    for i in range(n_req):
        n, h = stacks[i % 2]
        wl = rng.uniform(350, 1100)
        kp = k_parallel_from_angles(wl, rng.uniform(0, 60), rng.uniform(0, 90))
        pol = ('TE', 'TM', 'un')[i % 3]
        reqs.append(FilmRequest(n, h, wl, kp, 500.0, 3, pol=pol))
    return reqs


def _mixed_requests(n_req, seed=0):
    """Requests of different shapes: layer counts, order sets, periods, 1D/2D."""
    from emustack_b200.serving import FilmRequest
    from oracle.gsm_oracle import k_parallel_from_angles
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n_req):
        L = int(rng.integers(2, 13))
        n = np.concatenate([[1.46 + 0j], rng.uniform(1.3, 4.0, L - 2) + 1j * rng.uniform(0, 0.5, L - 2),
                            [1.0 + 0j]])
        mo = int(rng.integers(1, 7))
        per = float(rng.choice([500.0, 600.0, 700.0]))
        w1d = bool(rng.random() < 0.25)
        wl = rng.uniform(350, 1100)
        kp = k_parallel_from_angles(wl, rng.uniform(0, 60), rng.uniform(0, 90))
        reqs.append(FilmRequest(n, rng.uniform(20, 300, L - 2), wl, kp, per, mo,
                                pol=('TE', 'TM', 'un', 'R Circ')[i % 4], world_1d=w1d))
    return reqs


def _alone_var(req):
    from emustack_b200.films import FilmVarSolver
    s = FilmVarSolver()
    pl = s.plan([req])
    out = s.solve(pl)
    return s.unpack(pl, {k: v.cpu().numpy() for k, v in out.items()})[0]


def _alone(req):
    from emustack_b200.films import FilmStackSolver
    s = FilmStackSolver(len(req.n), req.max_order, req.period)
    dev = s.device
    o = s.solve(torch.tensor([req.wl_nm], dtype=torch.float64, device=dev),
                torch.tensor(req.k_pll.reshape(1, 2), device=dev),
                torch.tensor(req.n.reshape(1, -1), device=dev), torch.tensor(req.heights, device=dev),
                pol=req.pol)
    return {k: v[0].cpu().numpy() for k, v in o.items()}


def test_mixed_shapes_same_alone_and_in_the_mix():
    """Requests of different shapes share launches; each result equals the
    same request solved alone, bit for bit."""
    from emustack_b200.serving import GsmServer
    reqs = _mixed_requests(500)
    with GsmServer(max_batch=96) as srv:
        futs = []
        for i, r in enumerate(reqs):
            futs.append(srv.submit(r))
            if i % 40 == 0:
                time.sleep(0.002)  # arrivals while batches run
        res = [f.result(timeout=120) for f in futs]
        st = srv.stats()
    assert st['requests'] == len(reqs) and st['batches'] > 4
    assert len({r.signature for r in reqs}) > 50
    for i in range(0, len(reqs), 23):
        a = _alone_var(reqs[i])
        for k in ('R_net', 'T_net', 'a_list', 't_list', 'r_list', 'flags', 'specular'):
            assert np.array_equal(res[i][k], a[k]), (i, k)


def test_results_same_alone_and_in_the_mix():
    from emustack_b200.serving import GsmServer
    reqs = _requests(600)
    with GsmServer(max_batch=128, batching='grouped') as srv:
        futs = []
        for i, r in enumerate(reqs):
            futs.append(srv.submit(r))
            if i % 50 == 0:
                time.sleep(0.002)  # arrivals while batches run
        res = [f.result(timeout=120) for f in futs]
        st = srv.stats()
    assert st['requests'] == len(reqs)
    assert st['batches'] > 4
    assert np.isfinite(st['p99_ms'])
    for i in list(range(0, len(reqs), 37)):
        a = _alone(reqs[i])
        for k in ('R_net', 'T_net', 'a_list', 't_list', 'r_list'):
            assert np.array_equal(res[i][k], a[k]), (i, k)


def test_serving_matches_oracle():
    from emustack_b200.serving import GsmServer
    from oracle import gsm_oracle as O
    reqs = _requests(40, seed=1) + _mixed_requests(20, seed=5)
    with GsmServer(max_batch=16) as srv:
        futs = [srv.submit(r) for r in reqs]
        res = [f.result(timeout=120) for f in futs]
    for r, o in zip(reqs[::7], res[::7]):
        ref = O.film_stack_point(r.n, r.heights, r.wl_nm, r.k_pll, r.period, r.period_y, r.max_order,
                                 r.world_1d, pol=r.pol)
        np.testing.assert_allclose(o['R_net'], np.diag(ref.R_net), rtol=1e-9, atol=1e-10)
        if not o['flags'] & 4:
            np.testing.assert_allclose(o['a_list'], np.asarray(ref.a_list, float), rtol=1e-9, atol=1e-10)


def test_admission_respects_hbm_budget():
    from emustack_b200.serving import GsmServer
    reqs = _requests(400, seed=2)[::2]   # one stack shape: equal device footprint per request
    per = reqs[0].bytes_on_device()
    assert all(r.bytes_on_device() == per for r in reqs)
    for mode in ('mixed', 'grouped'):
        with GsmServer(max_batch=1000, hbm_budget_bytes=10 * per, batching=mode) as srv:
            futs = [srv.submit(r) for r in reqs]
            [f.result(timeout=120) for f in futs]
            assert max(srv.batch_sizes) <= 10
