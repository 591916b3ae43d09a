"""GPU parity of the 1D-grating overlap path against the oracle
(oracle/overlap1d_oracle.py, a restatement of J_overlap_1d.f,
J_dagger_overlap_1d.f, pw_ordering_1d.f + z_indexx.f, pw_matrix_1d_to_2d.f,
orthogonal_1d.f and normalisation_1d.f).

The kernels evaluate the element integrals of P2 / P3 x exp(-+ i alpha x)
from power series / recurrences of the moments int t^k exp(i theta t); the
oracle by Gauss-Legendre quadrature.  Both are the exact integrals to
rounding, so J, J_dag and the orthogonality matrix are held to 1e-12 of the
largest entry.  Stacks built from the kernels' J are held to the
1e-9 bar of the other dense tests against the oracle's chain.
"""
import numpy as np
import pytest
import torch

from oracle import gsm_oracle as G
from oracle import overlap1d_oracle as O

pytestmark = pytest.mark.gpu


def _mesh(n_el, seed, types=None):
    from emustack_b200.mesh import Mesh1D
    return Mesh1D.uniform(n_el, jitter=0.6, seed=seed, types=types)


def _fields(rng, nel, M, scale=1.0):
    s = rng.standard_normal((nel, M, 11)) + 1j * rng.standard_normal((nel, M, 11))
    return scale * s


def _close(got, ref, rel=1e-12, msg=''):
    got, ref = np.asarray(got), np.asarray(ref)
    np.testing.assert_allclose(got, ref, rtol=0, atol=rel * max(1.0, np.abs(ref).max()), err_msg=msg)


@pytest.mark.parametrize('bx,by,max_order', [(0.0, 0.0, 4), (0.37, -0.21, 6), (-1.3, 0.0, 10),
                                             (2.9, 0.8, 3)])
def test_J_and_J_dag_match_the_oracle(bx, by, max_order):
    from emustack_b200.overlap import DeviceMesh1D, overlap_1d_batch
    rng = np.random.default_rng(int(1000 * abs(bx)) + max_order)
    mesh = _mesh(40, seed=max_order)
    M, B = 23, 2
    k0 = np.array([2 * np.pi / 0.9, 2 * np.pi / 1.7])
    bloch = np.array([[bx, by], [bx * 0.5, by]])
    s1 = [_fields(rng, mesh.nel, M) for _ in range(B)]
    s2 = [_fields(rng, mesh.nel, M) for _ in range(B)]
    dev = torch.device('cuda')
    dm = DeviceMesh1D(mesh, dev)
    J, Jd, J2, Jd2, inv, rows = overlap_1d_batch(
        dm, max_order, bloch, k0, torch.tensor(np.stack(s1), device=dev),
        torch.tensor(np.stack(s2), device=dev), embed_2d=True)
    for b in range(B):
        _, inv_o = O.pw_order_1d(max_order, 1.0, bloch[b, 0], bloch[b, 1], k0[b])
        np.testing.assert_array_equal(inv[b], inv_o)
        Jo = O.overlap_1d(s1[b], mesh.table_nod, mesh.x, 1.0, bloch[b, 0], bloch[b, 1], max_order, inv_o)
        Jdo = O.overlap_1d(s2[b], mesh.table_nod, mesh.x, 1.0, bloch[b, 0], bloch[b, 1], max_order, inv_o,
                           dagger=True)
        _close(J[b].cpu().numpy(), Jo, msg='J problem %d' % b)
        _close(Jd[b].cpu().numpy(), Jdo, msg='J_dag problem %d' % b)
        J2o, Jd2o, _ = O.pw_matrix_1d_to_2d(Jo, Jdo, 1.0, bloch[b, 0], bloch[b, 1], max_order, k0[b], inv_o)
        _close(J2[b].cpu().numpy(), J2o, msg='J_2d problem %d' % b)
        _close(Jd2[b].cpu().numpy(), Jd2o, msg='J_dag_2d problem %d' % b)


def test_orthogonality_matrix_and_normalisation_match_the_oracle():
    from emustack_b200.overlap import DeviceMesh1D, mode_overlap_1d
    rng = np.random.default_rng(12)
    mesh = _mesh(33, seed=2, types=(np.arange(33) % 3 == 1) + 1)
    M = 17
    s1, s2 = _fields(rng, mesh.nel, M), _fields(rng, mesh.nel, M)
    beta = rng.uniform(1, 9, M) + 1j * rng.uniform(0, 0.5, M)
    pp = np.array([1.0 + 0j, 2.25 - 0.1j])
    k0, by = 2 * np.pi / 1.2, 0.43
    dev = torch.device('cuda')
    dm = DeviceMesh1D(mesh, dev)
    args = (dm, pp, torch.tensor([k0], dtype=torch.float64, device=dev),
            torch.tensor([[0.1, by]], dtype=torch.float64, device=dev),
            torch.tensor(beta.reshape(1, M), device=dev), torch.tensor(s1[None], device=dev),
            torch.tensor(s2[None], device=dev))
    full = mode_overlap_1d(*args, full=True)[0].cpu().numpy()
    ref = O.overlap_matrix_1d(s1, s2, beta, mesh.table_nod, mesh.type_el, pp, mesh.x, k0, by)
    _close(full, ref, msg='overlap matrix')
    diag, scale, nsmall = mode_overlap_1d(*args)
    _close(diag[0].cpu().numpy(), np.diag(ref), msg='diagonal')
    assert int(nsmall[0]) == 0
    n1, _ = O.normalise_1d(s1, s2, ref)
    # the normalisation factor of mode m is the ratio of the normalised field to the field
    np.testing.assert_allclose(scale[0].cpu().numpy(), n1[0, :, 0] / s1[0, :, 0], rtol=1e-12)


def _stack_1d(seed, world_1d, swap=False):
    """A golden-case-4-shaped stack (period 760 nm, max order 6, two
    '1D_array' gratings of 46 Bloch modes between films), the gratings'
    J / J_dag from mode fields: drop-in objects and the oracle's chain."""
    from emustack_b200 import materials, objects
    rng = np.random.default_rng(seed)
    period, mo, wl = 760.0, 6, 800.0
    light = objects.Light(wl, max_order_PWs=mo, theta=0.0, phi=0.0)
    kp = light.k_pll
    air = G.make_air_ref(wl, kp, period, period, mo, world_1d)
    k0 = 2 * np.pi / G.wl_norm(wl, period)
    bx, by = np.asarray(kp) * period
    sub = objects.ThinFilm(period, height_nm='semi_inf', world_1d=world_1d,
                           material=materials.Material(1.46 + 0j), loss=False)
    sup = objects.ThinFilm(period, height_nm='semi_inf', world_1d=world_1d, material=materials.Air,
                           loss=False)
    lays = [sub.calc_modes(light)]
    olays = [G.film_layer(1.46 + 0j, wl, kp, period, air, None, period, mo, world_1d, False)]
    # two gratings with a film between them: in the 2D order set the orders
    # with py != 0 do not couple to a 1D grating (R12 = -1 for them), so two
    # gratings with only an air gap between them make those orders an
    # exactly singular cavity -- in the reference as here
    hs = [150.0, 80.0, 900.0]
    for li, h in enumerate(hs):
        if li == 1:
            nf = 2.1 + 0.05j
            f = objects.ThinFilm(period, height_nm=h, world_1d=world_1d, material=materials.Material(nf))
            lays.append(f.calc_modes(light))
            olays.append(G.film_layer(nf, wl, kp, period, air, h, period, mo, world_1d, True))
            continue
        mesh = _mesh(60, seed=int(h))
        M = 46
        kz = rng.uniform(0, 2 * k0, M) + 1j * rng.uniform(0, 0.1 * k0, M)
        s1 = _fields(rng, mesh.nel, M, 0.5)
        s2 = _fields(rng, mesh.nel, M, 0.5)
        if swap:
            # adjoint mode 3 made orthogonal to prime mode 3: the pair swap runs
            ovl = O.overlap_matrix_1d(s1, s2, kz, mesh.table_nod, mesh.type_el, [1.0], mesh.x, k0, by)
            s2[:, 3] -= ovl[3, 3] / ovl[5, 3] * s2[:, 5]
        ns = objects.NanoStruct('1D_array', period, 190, height_nm=h, world_1d=world_1d, mesh=mesh)
        lays.append(ns.calc_modes(light, k_z=kz, fields=dict(sol1=s1, sol2=s2)))
        ovl, s2w, _ = O.orthogonal_1d(s1, s2, kz, mesh.table_nod, mesh.type_el, [1.0], mesh.x, k0, by)
        n1, n2 = O.normalise_1d(s1, s2w, ovl)
        _, inv = O.pw_order_1d(mo, mesh.period_x, bx, by, k0)
        J = O.overlap_1d(n1, mesh.table_nod, mesh.x, mesh.period_x, bx, by, mo, inv)
        Jd = O.overlap_1d(n2, mesh.table_nod, mesh.x, mesh.period_x, bx, by, mo, inv, dagger=True)
        if not world_1d:
            J, Jd, _ = O.pw_matrix_1d_to_2d(J, Jd, mesh.period_x, bx, by, mo, k0, inv)
        olays.append(G.OracleLayer('struct', kz, h, J=J, J_dag=Jd))
    lays.append(sup.calc_modes(light))
    olays.append(G.film_layer(1.0 + 0j, wl, kp, period, air, None, period, mo, world_1d, False))
    return lays, olays, air, hs, period


@pytest.mark.parametrize('world_1d,swap', [(True, False), (True, True), (False, False)])
def test_stack_of_1d_gratings_from_fields_matches_the_oracle(world_1d, swap):
    """Fields -> orthogonality, pair swaps, normalisation, J / J_dag (1D set,
    or embedded in the 2D set) -> interfaces -> cascade -> fluxes, through
    NanoStruct('1D_array').calc_modes(fields=...) and Stack.calc_scat."""
    from emustack_b200.stack import Stack
    lays, olays, air, hs, period = _stack_1d(5, world_1d, swap)
    for i in (1, 3):
        Jo = olays[i].J
        _close(lays[i].J, Jo, rel=1e-11, msg='layer %d J' % i)
        _close(lays[i].J_dag, olays[i].J_dag, rel=1e-11, msg='layer %d J_dag' % i)
    st = Stack(lays)
    st.calc_scat(pol='TE')
    ref = G.calc_scat(olays, air, period, pol='TE', heights_nm=hs)
    tol = dict(rtol=1e-9, atol=1e-9 * max(1.0, np.abs(ref.R_net).max()))
    np.testing.assert_allclose(st.R_net, ref.R_net, **tol)
    np.testing.assert_allclose(st.T_net, ref.T_net, **tol)
    for k in ('a_list', 't_list', 'r_list'):
        np.testing.assert_allclose(np.asarray(getattr(st, k), float), np.asarray(getattr(ref, k), float),
                                   rtol=1e-9, atol=1e-9, err_msg=k)
