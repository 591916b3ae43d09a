"""GPU parity of the uneven-batch film kernel (emu_film_var_batch).

One launch solves points of different shapes -- layer counts, order sets
(1D / 2D, max order, periods), polarisations, incoming vectors -- each of
which the reference solves with its own Stack(layers).calc_scat call
(backend/stack.py:162-426).  Checked against the golden fixtures, against
the CPU oracle and against the uniform film kernel point by point.
Tolerance: FP64 throughout, rtol 1e-9 / atol 1e-10 against the oracle and
the fixtures.  Against the uniform kernel, R_net / T_net come from the same
per-order code and must agree bit for bit; the flux sums are accumulated
with shared-memory atomics in no fixed order, so a/t/r lists agree to 1e-13
(relative, and absolute for the near-zero absorptances that are differences
of order-one fluxes).
"""
import numpy as np
import pytest
import torch

from fixtures import film_inputs, load_points

pytestmark = pytest.mark.gpu

TOL = dict(rtol=1e-9, atol=1e-10)


def _host(out):
    return {k: v.cpu().numpy() for k, v in out.items()}


def _solve(points, **kw):
    from emustack_b200.films import FilmVarSolver
    s = FilmVarSolver()
    pl = s.plan(points)
    out = s.solve(pl, **kw)
    torch.cuda.synchronize()
    return pl, s.unpack(pl, _host(out))


def _golden_points():
    pts = []
    for name in ('case_0', 'films10', 'edge_cases'):
        gp, _ = load_points(name)
        for p, pt in enumerate(gp):
            fi = film_inputs(pt)
            if fi is None or fi['shears'] is not None:
                continue
            pts.append(('%s p%d' % (name, p), pt, fi))
    return pts


def _point(fi):
    from emustack_b200.films import FilmPoint
    return FilmPoint(fi['n'], fi['heights'], fi['wl'], fi['k_pll'], fi['period'], fi['max_order'],
                     pol=fi['pol'], period_y=fi['period_y'], world_1d=fi['world_1d'],
                     incoming=fi['incoming'])


def test_golden_points_in_one_launch():
    gp = _golden_points()
    assert len(gp) >= 10
    pl, res = _solve([_point(fi) for _, _, fi in gp], want_num_prop=True)
    for (msg, pt, fi), r in zip(gp, res):
        np.testing.assert_allclose(r['R_net'], np.diag(pt['R_net']), **TOL, err_msg=msg + ' R_net')
        np.testing.assert_allclose(r['T_net'], np.diag(pt['T_net']), **TOL, err_msg=msg + ' T_net')
        if r['flags'] & 4:
            assert np.all(pt['a_list'] == 0)
        else:
            np.testing.assert_allclose(r['a_list'], pt['a_list'], **TOL, err_msg=msg + ' a')
            np.testing.assert_allclose(r['t_list'], pt['t_list'], **TOL, err_msg=msg + ' t')
            np.testing.assert_allclose(r['r_list'], np.asarray(pt['r_list']).reshape(-1)[0], **TOL)
        for i, lay in enumerate(pt['layers']):
            assert r['specular'] == int(lay['specular_order'])
            assert int(r['num_prop'][i]) == int(lay['num_prop'])


def _random_points(rng, n):
    from emustack_b200.films import FilmPoint, grating_orders
    pols = ['TE', 'TM', 'un', 'R Circ', 'L Circ']
    pts = []
    for i in range(n):
        L = int(rng.integers(2, 11))
        w1d = bool(rng.random() < 0.3)
        mo = int(rng.integers(0, 6))
        per = float(rng.choice([400.0, 500.0, 600.0, 760.0]))
        per_y = per if w1d or rng.random() < 0.7 else float(rng.choice([380.0, 610.0]))
        wl = float(rng.uniform(350.0, 1200.0))
        th = float(rng.uniform(0, 0.6))
        kp = np.array([np.sin(th), 0.3 * np.sin(th)]) * 2 * np.pi / wl
        n = rng.uniform(1.0, 4.0, L) + 1j * rng.uniform(0, 0.3, L) * (rng.random(L) < 0.6)
        n[-1] = 1.0
        h = rng.uniform(5.0, 400.0, L - 2)
        inc = None
        if i % 7 == 3:
            npw = len(grating_orders(mo, per, per_y, w1d)[0])
            inc = np.zeros(2 * npw, complex)
            inc[rng.integers(0, 2 * npw, size=min(3, 2 * npw))] = rng.normal(size=min(3, 2 * npw))
        pts.append(FilmPoint(n, h, wl, kp, per, mo, pol=pols[i % 5], period_y=per_y,
                             world_1d=w1d, incoming=inc))
    return pts


def test_random_mixed_batch_matches_uniform_kernel_and_oracle():
    from emustack_b200.films import FilmStackSolver
    from oracle import gsm_oracle as O
    rng = np.random.default_rng(7)
    pts = _random_points(rng, 300)
    pl, res = _solve(pts)
    dev = torch.device('cuda')
    for i, (p, r) in enumerate(zip(pts, res)):
        L = len(p.n)
        s = FilmStackSolver(L, p.max_order, p.period, p.period_y, p.world_1d)
        inc = None if p.incoming is None else torch.tensor(p.incoming.reshape(1, -1), device=dev)
        o = s.solve(torch.tensor([p.wl_nm], dtype=torch.float64, device=dev),
                    torch.tensor(p.k_pll.reshape(1, 2), device=dev),
                    torch.tensor(p.n.reshape(1, L), device=dev),
                    torch.tensor(p.heights, device=dev) if L > 2 else None,
                    pol=p.pol, incoming=inc, want=('specular',))
        o = _host(o)
        msg = 'point %d' % i
        np.testing.assert_array_equal(r['R_net'], o['R_net'][0], err_msg=msg)
        np.testing.assert_array_equal(r['T_net'], o['T_net'][0], err_msg=msg)
        np.testing.assert_allclose(r['a_list'], o['a_list'][0], rtol=1e-13, atol=1e-13, err_msg=msg)
        np.testing.assert_allclose(r['t_list'], o['t_list'][0], rtol=1e-13, atol=1e-13, err_msg=msg)
        np.testing.assert_allclose(r['r_list'], o['r_list'][0], rtol=1e-13, atol=1e-13, err_msg=msg)
        assert r['flags'] == o['flags'][0] and r['specular'] == o['specular'][0]
        if i % 10 == 0:
            ref = O.film_stack_point(list(p.n), list(p.heights), p.wl_nm, p.k_pll, p.period,
                                     p.period_y, p.max_order, p.world_1d, pol=p.pol,
                                     incoming_amplitudes=p.incoming)
            np.testing.assert_allclose(r['R_net'], np.diag(ref.R_net), **TOL, err_msg=msg)
            np.testing.assert_allclose(r['T_net'], np.diag(ref.T_net), **TOL, err_msg=msg)
            if not r['flags'] & 4:
                np.testing.assert_allclose(r['a_list'], ref.a_list, **TOL, err_msg=msg)
                np.testing.assert_allclose(r['t_list'], ref.t_list, **TOL, err_msg=msg)


def test_bad_descriptor_is_flagged_and_skipped():
    """A point whose slices fall outside the packed arrays is not solved:
    it gets EMU_PT_BAD_POINT and the other points are unaffected."""
    from emustack_b200 import _lib
    from emustack_b200.films import FilmVarSolver
    rng = np.random.default_rng(3)
    pts = _random_points(rng, 12)
    s = FilmVarSolver()
    pl = s.plan(pts)
    good = s.unpack(pl, _host(s.solve(pl)))
    torch.cuda.synchronize()
    desc = pl.desc.copy()
    desc[5]['n_off'] = pl.n_len              # past the end of d_n
    desc[8]['n_layers'] = pl.max_layers + 1
    pl.h_desc.numpy()[:] = desc.view(np.uint8)
    out = _host(s.solve(pl))
    torch.cuda.synchronize()
    assert out['flags'][5] == _lib.PT_BAD_POINT and out['flags'][8] == _lib.PT_BAD_POINT
    bad = s.unpack(pl, out)
    for i in range(12):
        if i in (5, 8):
            continue
        np.testing.assert_array_equal(bad[i]['R_net'], good[i]['R_net'])
        assert bad[i]['flags'] == good[i]['flags']
