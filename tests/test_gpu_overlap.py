"""GPU parity of the overlap integrals J / J_dag and the Bloch-mode
normalisation against the C restatement of the reference Fortran
(oracle/overlap_oracle.c: J_overlap.f, J_dagger_overlap.f, pw_ordering.f,
orthogonal.f, normalisation.f).  FP64; rtol 1e-9 / atol 1e-11."""
import numpy as np
import pytest
import torch

from emustack_b200.mesh import square_cell
from oracle import overlap as OV

pytestmark = pytest.mark.gpu

TOL = dict(rtol=1e-9, atol=1e-11)


def _fields(rng, nel, nval):
    return (rng.standard_normal((nel, nval, 13, 3)) + 1j * rng.standard_normal((nel, nval, 13, 3)))


@pytest.mark.parametrize('n,dy,mo,nval,chunk', [(6, 1.0, 2, 7, 0), (5, 0.8, 1, 5, 7), (8, 1.0, 3, 33, 13)])
def test_overlap_matches_oracle(n, dy, mo, nval, chunk):
    from emustack_b200.films import grating_orders
    from emustack_b200.overlap import DeviceMesh, overlap_batch
    rng = np.random.default_rng(n * 10 + mo)
    mesh = square_cell(n, dy=dy, radius=0.3, jitter=0.3, seed=n)
    B = 2
    blochs = np.array([[0.21, -0.37], [0.05, 0.44]])
    k0s = 2 * np.pi / np.array([0.9, 1.37])
    s1 = np.stack([_fields(rng, mesh.nel, nval) for _ in range(B)])
    s2 = np.stack([_fields(rng, mesh.nel, nval) for _ in range(B)])
    px, py = grating_orders(mo, 600.0, 600.0 * dy)
    dm = DeviceMesh(mesh)
    area = dy
    J, Jd, inv = overlap_batch(dm, px, py, mo, torch.tensor(blochs, device='cuda'),
                               torch.tensor(k0s, device='cuda'), torch.tensor(s1, device='cuda'),
                               torch.tensor(s2, device='cuda'), area_norm=area, dy=dy,
                               elements_per_chunk=chunk)
    for b in range(B):
        oinv, opx, opy = OV.pw_ordering(mo, 1.0, dy, blochs[b], k0s[b])
        np.testing.assert_array_equal(opx, px)
        np.testing.assert_array_equal(opy, py)
        np.testing.assert_array_equal(inv[b].cpu().numpy(), oinv)
        Jo = OV.J_overlap(mesh.x, mesh.table_nod, s1[b], 1.0, dy, blochs[b], oinv, mo) / area
        Jdo = OV.J_dagger_overlap(mesh.x, mesh.table_nod, s2[b], 1.0, dy, blochs[b], oinv, mo)
        np.testing.assert_allclose(J[b].cpu().numpy(), Jo, **TOL)
        np.testing.assert_allclose(Jd[b].cpu().numpy(), Jdo, **TOL)


def test_normalisation_matches_oracle():
    from emustack_b200.overlap import DeviceMesh, mode_normalisation
    rng = np.random.default_rng(5)
    mesh = square_cell(5, radius=0.3, jitter=0.25)
    nval = 9
    s1, s2 = _fields(rng, mesh.nel, nval), _fields(rng, mesh.nel, nval)
    b1 = rng.uniform(1, 3, nval) + 1j * rng.uniform(0, 0.1, nval)
    pp = np.array([1.0 + 0j, 0.7 + 0.1j])
    k0 = 2 * np.pi / 1.1
    ovl, perm, scale, warn, s2n, b2 = OV.orthogonal_normalise(mesh.x, mesh.table_nod, mesh.type_el, pp, b1,
                                                              b1, s1, s2, k0)
    dm = DeviceMesh(mesh)
    diag, sc, ns = mode_normalisation(dm, pp, torch.tensor([k0], dtype=torch.float64, device='cuda'),
                                      torch.tensor(b1[None], device='cuda'),
                                      torch.tensor(s1[None], device='cuda'), torch.tensor(s2[None], device='cuda'))
    assert int(ns[0]) == 0
    np.testing.assert_allclose(diag[0].cpu().numpy(), np.diag(ovl), rtol=1e-10)
    np.testing.assert_allclose(sc[0].cpu().numpy(), scale, rtol=1e-10)


def test_simmo_from_fields_stack_matches_oracle():
    """A nanostructured layer built from mode fields: GPU normalisation + J /
    J_dag + interface + cascade against the oracle chain."""
    from emustack_b200 import objects, materials
    from emustack_b200.stack import Stack
    from oracle import gsm_oracle as O
    rng = np.random.default_rng(6)
    period = 600.0
    mesh = square_cell(6, radius=0.2)
    light = objects.Light(780.0, max_order_PWs=2, theta=8.0, phi=25.0)
    nval = 30
    s1, s2 = 0.05 * _fields(rng, mesh.nel, nval), 0.05 * _fields(rng, mesh.nel, nval)
    k0 = 2 * np.pi / (780.0 / period)
    kz = rng.uniform(0, 2 * k0, nval) + 1j * rng.uniform(0, 0.1 * k0, nval)
    ns = objects.NanoStruct('2D_array', period, 240, height_nm=90.0, mesh=mesh)
    sim = ns.calc_modes(light, k_z=kz, fields=dict(sol1=s1, sol2=s2, beta1=kz))
    sub = objects.ThinFilm(period, height_nm='semi_inf', material=materials.Material(1.46 + 0j), loss=False)
    sup = objects.ThinFilm(period, height_nm='semi_inf', material=materials.Air, loss=False)
    st = Stack([sub.calc_modes(light), sim, sup.calc_modes(light)])
    st.calc_scat(pol='TE')
    # oracle chain
    air = O.make_air_ref(780.0, light.k_pll, period, period, 2)
    ovl, perm, scale, warn, s2n, b2 = OV.orthogonal_normalise(mesh.x, mesh.table_nod, mesh.type_el, [1.0, 1.0],
                                                              kz, kz, s1, s2, k0)
    inv, _, _ = OV.pw_ordering(2, 1.0, 1.0, air.k_pll_norm(), k0)
    J = OV.J_overlap(mesh.x, mesh.table_nod, s1, 1.0, 1.0, air.k_pll_norm(), inv, 2)
    Jd = OV.J_dagger_overlap(mesh.x, mesh.table_nod, s2n, 1.0, 1.0, air.k_pll_norm(), inv, 2)
    np.testing.assert_allclose(sim.J, J, **TOL)
    np.testing.assert_allclose(sim.J_dag, Jd, rtol=1e-9, atol=1e-10)
    layers = [O.film_layer(1.46, 780.0, light.k_pll, period, air, None, loss=False, max_order=2),
              O.OracleLayer('struct', kz, 90.0, J=J, J_dag=Jd),
              O.film_layer(1.0, 780.0, light.k_pll, period, air, None, loss=False, max_order=2)]
    r = O.calc_scat(layers, air, period, pol='TE', heights_nm=[90.0])
    np.testing.assert_allclose(st.R_net, r.R_net, rtol=1e-8, atol=1e-9)
    np.testing.assert_allclose(np.asarray(st.a_list, float), np.asarray(r.a_list, float), rtol=1e-8, atol=1e-9)


def test_pair_reordering_on_gpu_matches_oracle():
    """A vanishing <m|m> triggers the conjugate-pair swap loop of
    orthogonal.f:252-301 on the GPU: permutation, recomputed diagonal,
    normalisation factors and the J_dag built from them match the oracle."""
    from emustack_b200.films import grating_orders
    from emustack_b200.overlap import DeviceMesh, mode_normalisation, mode_reorder, overlap_batch
    rng = np.random.default_rng(21)
    mesh = square_cell(4, radius=0.3)
    nval = 5
    s1, s2 = _fields(rng, mesh.nel, nval), _fields(rng, mesh.nel, nval)
    s2[:, 1] = 0.0
    b1 = rng.uniform(1, 3, nval) + 0j
    k0 = 2 * np.pi / 0.95
    pp = [1.0 + 0j, 1.0 + 0j]
    ovl, perm, scale, warn, s2n, b2 = OV.orthogonal_normalise(mesh.x, mesh.table_nod, mesh.type_el, pp, b1, b1,
                                                              s1, s2, k0)
    assert list(perm) != list(range(nval))
    dm = DeviceMesh(mesh)
    args = (dm, pp, torch.tensor([k0], dtype=torch.float64, device='cuda'), torch.tensor(b1[None], device='cuda'),
            torch.tensor(s1[None], device='cuda'), torch.tensor(s2[None], device='cuda'))
    diag, sc, ns = mode_normalisation(*args)
    assert int(ns[0]) >= 1
    gperm, gdiag, gscale, gwarn = mode_reorder(*args)
    np.testing.assert_array_equal(gperm[0].cpu().numpy(), perm)
    np.testing.assert_allclose(gdiag[0].cpu().numpy(), np.diag(ovl), rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(gscale[0].cpu().numpy(), scale, rtol=1e-10)
    assert int(gwarn[0]) == warn
    mo = 1
    px, py = grating_orders(mo, 600.0, 600.0)
    bl = np.array([0.11, 0.07])
    J, Jd, inv = overlap_batch(dm, px, py, mo, torch.tensor(bl[None], device='cuda'),
                               torch.tensor([k0], dtype=torch.float64, device='cuda'), None,
                               torch.tensor(s2[None], device='cuda'), scale2=gscale, perm2=gperm)
    oinv, _, _ = OV.pw_ordering(mo, 1.0, 1.0, bl, k0)
    Jdo = OV.J_dagger_overlap(mesh.x, mesh.table_nod, s2n, 1.0, 1.0, bl, oinv, mo)
    np.testing.assert_allclose(Jd[0].cpu().numpy(), Jdo, rtol=1e-9, atol=1e-11)


@pytest.mark.parametrize('name', ['4testing-600_120.mail', '4testing-940_266_sq.mail'])
def test_reference_meshes_match_oracle(name):
    """J, J_dag and the adjoint normalisation on the reference's own test
    meshes (read with Mesh.from_mail: 518 and 2 528 P2 triangles, two
    material types), FP64 path against the C restatement."""
    from fixtures import reference_mesh
    from emustack_b200.films import grating_orders
    from emustack_b200.overlap import DeviceMesh, mode_normalisation, overlap_batch
    mesh = reference_mesh(name)
    rng = np.random.default_rng(mesh.nel)
    nval, mo = 12, 3
    s1, s2 = _fields(rng, mesh.nel, nval), _fields(rng, mesh.nel, nval)
    bloch, k0 = np.array([0.013, -0.021]), 2 * np.pi / 1.3
    px, py = grating_orders(mo, 600.0, 600.0)
    dm = DeviceMesh(mesh)
    J, Jd, inv = overlap_batch(dm, px, py, mo, torch.tensor(bloch[None], device='cuda'),
                               torch.tensor([k0], dtype=torch.float64, device='cuda'),
                               torch.tensor(s1[None], device='cuda'),
                               torch.tensor(s2[None], device='cuda'))
    oinv, _, _ = OV.pw_ordering(mo, 1.0, 1.0, bloch, k0)
    np.testing.assert_array_equal(inv[0].cpu().numpy(), oinv)
    Jo = OV.J_overlap(mesh.x, mesh.table_nod, s1, 1.0, 1.0, bloch, oinv, mo)
    Jdo = OV.J_dagger_overlap(mesh.x, mesh.table_nod, s2, 1.0, 1.0, bloch, oinv, mo)
    np.testing.assert_allclose(J[0].cpu().numpy(), Jo, **TOL)
    np.testing.assert_allclose(Jd[0].cpu().numpy(), Jdo, **TOL)
    b1 = rng.uniform(1, 3, nval) + 1j * rng.uniform(0, 0.1, nval)
    pp = np.array([1.0 + 0j, 3.5 ** 2 + 0.07j])
    ovl, perm, scale, warn, s2n, b2 = OV.orthogonal_normalise(mesh.x, mesh.table_nod, mesh.type_el, pp, b1,
                                                              b1, s1, s2, k0)
    diag, sc, ns = mode_normalisation(dm, pp, torch.tensor([k0], dtype=torch.float64, device='cuda'),
                                      torch.tensor(b1[None], device='cuda'), torch.tensor(s1[None], device='cuda'),
                                      torch.tensor(s2[None], device='cuda'))
    np.testing.assert_allclose(diag[0].cpu().numpy(), np.diag(ovl), rtol=1e-10)
    np.testing.assert_allclose(sc[0].cpu().numpy(), scale, rtol=1e-10)


@pytest.mark.parametrize('precision', ['fp64', 'tf32x3'])
def test_quadratic_fields_known_answer_gpu(precision):
    """Fields quadratic over the cell on the reference's 518-triangle mesh:
    J against the exact cell integrals (the quadrature error bound of the
    16-point rule per max order; the tensor-core path adds its split-TF32
    error, <= 5e-6 of max |J|)."""
    from fixtures import QUAD_BOUND, exact_J, quadratic_fields, reference_mesh
    from emustack_b200.films import grating_orders
    from emustack_b200.overlap import DeviceMesh, overlap_batch
    mesh = reference_mesh('4testing-600_120.mail')
    rng = np.random.default_rng(4)
    sol, Cf = quadratic_fields(mesh, 5, rng)
    bloch, k0 = np.array([0.31, -0.17]), 2 * np.pi / 1.1
    dm = DeviceMesh(mesh)
    for mo, bound in QUAD_BOUND.items():
        px, py = grating_orders(mo, 600.0, 600.0)
        J, _, inv = overlap_batch(dm, px, py, mo, torch.tensor(bloch[None], device='cuda'),
                                  torch.tensor([k0], dtype=torch.float64, device='cuda'),
                                  torch.tensor(sol[None], device='cuda'),
                                  torch.tensor(sol[None], device='cuda'), precision=precision)
        Je = exact_J(Cf, px, py, bloch, 1.0, 1.0, (0.0, 1.0, -1.0, 0.0), inv[0].cpu().numpy())
        tol = bound + (5e-6 if precision == 'tf32x3' else 0.0)
        err = np.abs(J[0].cpu().numpy() - Je).max() / np.abs(Je).max()
        assert err <= tol, (mo, err)
