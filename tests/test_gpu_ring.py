"""The device-resident request loop (emu_film_ring_*, serving.DeviceFilmServer).

A persistent kernel serves all-film spectral points that the host writes
into a ring of pinned, device-mapped slots.  Each request's results must
equal those of the uneven one-launch batch (emu_film_var_batch: the same
per-point recursion, one warp per point) -- per-order values bit for bit,
flux sums to rounding -- and the oracle's (a restatement of the reference's
FP64 GSM, backend/stack.py:162-426) at 1e-9.  The loop ends by itself when
idle and restarts on the next submit.  Each test stops its server before any
other device work (a running loop holds every SM).
"""
import time

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _requests(n, seed, max_mo=12, period=500.0):
    from emustack_b200.films import grating_orders
    from emustack_b200.serving import FilmRequest
    rng = np.random.default_rng(seed)
    pols = ('TE', 'TM', 'un', 'R Circ', 'L Circ')
    out = []
    for i in range(n):
        mo = int(rng.integers(0, max_mo + 1))
        L = int(rng.integers(2, 15))
        nn = np.concatenate([[1.46 + 0j], rng.uniform(1.3, 4.0, L - 2) + 1j * rng.uniform(0, 0.5, L - 2),
                             [1.0 + 0j]])
        wl = rng.uniform(350, 1100)
        th, ph = np.radians(rng.uniform(0, 60)), np.radians(rng.uniform(0, 90))
        k = 2 * np.pi / wl
        kp = np.array([k * np.sin(th) * np.cos(ph), k * np.sin(th) * np.sin(ph)])
        assert len(grating_orders(mo, period, period)[0]) <= 512
        out.append(FilmRequest(nn, rng.uniform(20, 300, L - 2), wl, kp, period, mo, pol=pols[i % 5]))
    return out


def _var_results(reqs):
    from emustack_b200.films import FilmVarSolver
    vs = FilmVarSolver(torch.device('cuda'))
    pl = vs.plan(reqs)
    out = vs.solve(pl)
    host = vs.fetch(out)
    torch.cuda.synchronize()
    return [{k: np.array(v) for k, v in r.items()} for r in vs.unpack(pl, host)]


def test_ring_matches_the_uneven_batch_and_the_oracle():
    from emustack_b200.serving import DeviceFilmServer
    from oracle import gsm_oracle as O
    reqs = _requests(700, seed=3)
    srv = DeviceFilmServer(capacity=256, idle_seconds=0.5)
    try:
        tickets = [srv.submit(r) for r in reqs]     # more requests than slots: reads free them
        got = [srv.take(t) for t in tickets]
        assert srv.stop() == 0
    finally:
        srv.close()
    ref = _var_results(reqs)
    for i, (g, v) in enumerate(zip(got, ref)):
        np.testing.assert_array_equal(g['R_net'], np.asarray(v['R_net']), err_msg='request %d' % i)
        np.testing.assert_array_equal(g['T_net'], np.asarray(v['T_net']), err_msg='request %d' % i)
        np.testing.assert_allclose(g['a_list'], np.asarray(v['a_list']), rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(g['t_list'], np.asarray(v['t_list']), rtol=1e-12, atol=1e-14)
        assert g['flags'] == int(v['flags'])
    for i in range(0, len(reqs), 70):
        r = reqs[i]
        o = O.film_stack_point(r.n, r.heights, r.wl_nm, r.k_pll, r.period, max_order=r.max_order, pol=r.pol)
        np.testing.assert_allclose(got[i]['R_net'], np.diag(o.R_net), rtol=1e-9, atol=1e-10)
        np.testing.assert_allclose(got[i]['a_list'], np.asarray(o.a_list, float), rtol=1e-9, atol=1e-10)


def test_ring_ends_when_idle_and_restarts_on_submit():
    from emustack_b200.serving import DeviceFilmServer
    reqs = _requests(40, seed=4, max_mo=5)
    srv = DeviceFilmServer(capacity=64, idle_seconds=0.2)
    try:
        first = [srv.take(srv.submit(r)) for r in reqs[:20]]
        deadline = time.time() + 5.0
        while srv.running() and time.time() < deadline:
            time.sleep(0.05)
        assert not srv.running()                     # ended by itself after 0.2 s idle
        second = [srv.take(srv.submit(r)) for r in reqs[20:]]
        assert srv.stop() == 0
    finally:
        srv.close()
    ref = _var_results(reqs)
    for g, v in zip(first + second, ref):
        np.testing.assert_array_equal(g['R_net'], np.asarray(v['R_net']))


def test_ring_refuses_requests_it_cannot_hold():
    from emustack_b200 import _lib
    from emustack_b200.serving import DeviceFilmServer, FilmRequest
    srv = DeviceFilmServer(capacity=8, idle_seconds=0.2)
    try:
        too_many_layers = FilmRequest(np.full(17, 1.5 + 0j), np.full(15, 50.0), 600.0, np.zeros(2), 500.0, 2)
        with pytest.raises(_lib.EmuError):
            srv.submit(too_many_layers)
        too_many_orders = FilmRequest(np.full(4, 1.5 + 0j), np.full(2, 50.0), 600.0, np.zeros(2), 500.0, 14)
        with pytest.raises(_lib.EmuError):
            srv.submit(too_many_orders)
        assert srv.stop() == 0
    finally:
        srv.close()


def test_poll_returns_results_read_early_to_free_slots():
    """More submissions than slots with nothing read: submit frees slots by
    reading the oldest results itself; poll / wait must still return every
    ticket's result exactly once, and ready() never consumes one."""
    from emustack_b200 import _lib
    from emustack_b200.serving import DeviceFilmServer
    reqs = _requests(60, seed=5, max_mo=4)
    srv = DeviceFilmServer(capacity=16, idle_seconds=0.5)
    try:
        tickets = [srv.submit(r) for r in reqs]
        got = {}
        deadline = time.time() + 30.0
        while len(got) < len(tickets) and time.time() < deadline:
            for t in tickets:
                if t not in got:
                    res = srv.poll(t)
                    if res is not None:
                        got[t] = res
        assert len(got) == len(tickets)
        with pytest.raises(_lib.EmuError):
            srv.poll(tickets[-1])                   # read once only
        assert srv.stop() == 0
    finally:
        srv.close()
    ref = _var_results(reqs)
    for t, v in zip(tickets, ref):
        np.testing.assert_array_equal(got[t]['R_net'], np.asarray(v['R_net']))


def test_batched_submit_and_poll_match_the_single_calls():
    """submit_many / poll_many (one library call per batch) return what the
    one-request calls return, bit for bit, also when a batch is larger than
    the free slots (the oldest results are then read to make room)."""
    from emustack_b200.serving import DeviceFilmServer
    reqs = _requests(90, seed=6, max_mo=6)
    srv = DeviceFilmServer(capacity=32, idle_seconds=0.5)
    try:
        tickets = srv.submit_many(reqs[:70])          # more than the 32 slots
        tickets += srv.submit_many(reqs[70:])
        assert len(tickets) == len(reqs) and len(set(tickets)) == len(reqs)
        got = {}
        deadline = time.time() + 30.0
        while len(got) < len(tickets) and time.time() < deadline:
            got.update(srv.poll_many([t for t in tickets if t not in got][:40]))
        assert len(got) == len(tickets)
        assert srv.stop() == 0
    finally:
        srv.close()
    ref = _var_results(reqs)
    for t, v in zip(tickets, ref):
        np.testing.assert_array_equal(got[t]['R_net'], np.asarray(v['R_net']))
        np.testing.assert_array_equal(got[t]['T_net'], np.asarray(v['T_net']))
        np.testing.assert_array_equal(got[t]['a_list'], np.asarray(v['a_list']))
        assert got[t]['flags'] == int(v['flags'])
