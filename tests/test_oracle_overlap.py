"""Known-answer tests pinning the C restatement of the overlap integrals
(oracle/overlap_oracle.c): no golden vector of the reference covers J or
J_dag (its stored results keep only the interface matrices), so the oracle
is checked against closed forms and exact symmetries of the reference's
formulas (backend/fortran/J_overlap.f, J_dagger_overlap.f, pw_ordering.f,
orthogonal.f, normalisation.f)."""
import numpy as np
import pytest

from emustack_b200.mesh import square_cell
from oracle import overlap as OV


def _fields(rng, nel, nval, real=False):
    s = rng.standard_normal((nel, nval, 13, 3))
    if not real:
        s = s + 1j * rng.standard_normal((nel, nval, 13, 3))
    return s.astype(np.complex128)


def test_constant_field_matches_closed_form():
    """A field constant in x gives J_E = beta/|k| * int_cell exp(-i k.x) and
    J_K = alpha/|k| * int_cell exp(-i k.x); the cell integral is
    (1 - e^{-i alpha})/(i alpha) * (1 - e^{-i beta dy})/(i beta)."""
    dy = 1.0
    mesh = square_cell(32, dy=dy)
    nel = mesh.nel
    sol = np.zeros((nel, 1, 13, 3), np.complex128)
    sol[:, 0, :6, 0] = 1.0
    bloch = np.array([0.3, 0.17])
    k0 = 2 * np.pi / 1.3
    inv, px, py = OV.pw_ordering(2, 1.0, dy, bloch, k0)
    J = OV.J_overlap(mesh.x, mesh.table_nod, sol, 1.0, dy, bloch, inv, 2)
    npw = len(inv)
    for s in range(npw):
        a = bloch[0] + 2 * np.pi * px[s]
        b = bloch[1] + 2 * np.pi * py[s] / dy
        ix = (1 - np.exp(-1j * a)) / (1j * a)
        iy = (1 - np.exp(-1j * b * dy)) / (1j * b)
        nrm = 1 / np.hypot(a, b)
        np.testing.assert_allclose(J[inv[s], 0], b * nrm * ix * iy, atol=2e-7)
        np.testing.assert_allclose(J[npw + inv[s], 0], a * nrm * ix * iy, atol=2e-7)


def test_dagger_is_conjugate_transpose_for_real_fields():
    """Only the sign of the exponent differs (J_overlap.f:144 vs
    J_dagger_overlap.f:142): for real fields J_dag = conj(J)^T exactly."""
    rng = np.random.default_rng(1)
    mesh = square_cell(5, dy=0.8, radius=0.25, jitter=0.3)
    sol = _fields(rng, mesh.nel, 4, real=True)
    bloch = np.array([0.21, -0.4])
    inv, px, py = OV.pw_ordering(2, 1.0, 0.8, bloch, 2 * np.pi / 0.9)
    J = OV.J_overlap(mesh.x, mesh.table_nod, sol, 1.0, 0.8, bloch, inv, 2)
    Jd = OV.J_dagger_overlap(mesh.x, mesh.table_nod, sol, 1.0, 0.8, bloch, inv, 2)
    np.testing.assert_allclose(Jd, J.conj().T, rtol=1e-14, atol=1e-15)


def test_element_renumbering_invariance():
    rng = np.random.default_rng(2)
    mesh = square_cell(4, radius=0.3, jitter=0.2)
    sol = _fields(rng, mesh.nel, 3)
    bloch = np.array([0.1, 0.05])
    inv, _, _ = OV.pw_ordering(1, 1.0, 1.0, bloch, 2 * np.pi / 1.7)
    J = OV.J_overlap(mesh.x, mesh.table_nod, sol, 1.0, 1.0, bloch, inv, 1)
    perm = rng.permutation(mesh.nel)
    J2 = OV.J_overlap(mesh.x, mesh.table_nod[perm], sol[perm], 1.0, 1.0, bloch, inv, 1)
    np.testing.assert_allclose(J2, J, rtol=1e-12, atol=1e-13)


def test_pw_ordering_matches_air_sort():
    """The Fortran sort key -Re(kz^2) orders plane waves as the air
    reference's argsort(-Re kz + Im kz) does (backend/mode_calcs.py:170)."""
    from oracle import gsm_oracle as O
    for wl, mo, kp in ((600.0, 3, (1.234e-4, 0.53e-4)), (913.0, 4, (3.1e-3, -1.07e-3))):
        per = 600.0
        air = O.make_air_ref(wl, np.array(kp), per, per, mo)
        inv, px, py = OV.pw_ordering(mo, 1.0, 1.0, air.k_pll_norm(), 2 * np.pi / O.wl_norm(wl, per))
        rx, ry = O.grating_orders_2d(mo, per, per)
        np.testing.assert_array_equal(px, rx)
        np.testing.assert_array_equal(py, ry)
        np.testing.assert_array_equal(np.argsort(inv), air.sort_order)


def test_normalisation_scales_adjoint_modes():
    rng = np.random.default_rng(3)
    mesh = square_cell(3, radius=0.3)
    nval = 4
    s1, s2 = _fields(rng, mesh.nel, nval), _fields(rng, mesh.nel, nval)
    b1 = rng.uniform(1, 3, nval) + 1j * rng.uniform(0, 0.1, nval)
    ovl, perm, scale, warn, s2n, b2 = OV.orthogonal_normalise(mesh.x, mesh.table_nod, mesh.type_el,
                                                              [1.0, 1.0], b1, b1, s1, s2, 2 * np.pi / 1.1)
    assert warn == 0 and (perm == np.arange(nval)).all()
    np.testing.assert_allclose(scale, 1 / np.sqrt(np.diag(ovl)) ** 2)
    # the normalised adjoint modes give a unit diagonal
    ovl2, _, scale2, _, _, _ = OV.orthogonal_normalise(mesh.x, mesh.table_nod, mesh.type_el, [1.0, 1.0],
                                                       b1, b1, s1, s2n, 2 * np.pi / 1.1)
    np.testing.assert_allclose(np.diag(ovl2), 1.0, rtol=1e-12)


def test_pair_reordering_swaps_adjoint_modes():
    """A vanishing diagonal entry triggers the conjugate-pair swap of
    orthogonal.f:252-301: the adjoint mode is exchanged with every later
    mode it overlaps, then the matrix is recomputed."""
    rng = np.random.default_rng(4)
    mesh = square_cell(3)
    nval = 3
    s1, s2 = _fields(rng, mesh.nel, nval), _fields(rng, mesh.nel, nval)
    s2[:, 0] = 0.0
    b1 = np.ones(nval, np.complex128)
    ovl, perm, scale, warn, s2n, b2 = OV.orthogonal_normalise(mesh.x, mesh.table_nod, mesh.type_el,
                                                              [1.0], b1, b1 * np.arange(1, 4), s1, s2, 5.0)
    # mode 0 is swapped with 1 then with 2 (both overlap prime mode 0)
    assert list(perm) == [2, 0, 1]
    np.testing.assert_allclose(b2, [3, 1, 2])


@pytest.mark.parametrize('name', ['4testing-600_120.mail', '4testing-940_266_sq.mail'])
def test_quadratic_fields_known_answer_on_reference_meshes(name):
    """Fields that are quadratic polynomials over the cell, on the
    reference's own test meshes (read by Mesh.from_mail): the oracle's J
    (16-point rule, degree 8, on each element) against the exact cell
    integrals of polynomial x plane wave; the difference is the quadrature
    error, bounded per max order."""
    from fixtures import QUAD_BOUND, exact_J, quadratic_fields, reference_mesh
    mesh = reference_mesh(name)
    rng = np.random.default_rng(len(name))
    sol, Cf = quadratic_fields(mesh, 3, rng)
    bloch, k0 = np.array([0.31, -0.17]), 2 * np.pi / 1.1
    for mo, bound in QUAD_BOUND.items():
        inv, px, py = OV.pw_ordering(mo, 1.0, 1.0, bloch, k0)
        Jo = OV.J_overlap(mesh.x, mesh.table_nod, sol, 1.0, 1.0, bloch, inv, mo)
        Je = exact_J(Cf, px, py, bloch, 1.0, 1.0, (0.0, 1.0, -1.0, 0.0), inv)
        assert np.abs(Jo - Je).max() <= bound * np.abs(Je).max(), (mo, np.abs(Jo - Je).max())
