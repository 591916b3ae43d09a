"""GPU parity of the 1D FEM Bloch-mode solve (emustack_b200.fem.FemMesh1D,
csrc/fem.cu: emu_fem1d_*), on the two gratings of the reference's test
case 4 with the meshes and inputs the reference passes to its solver
(tests/golden/fem1d.npz; the centre inclusion given the width of the
reference's stored run, as tests/test_oracle_fem1d.py explains):

* element matrices and assembly against the oracle (oracle/fem1d_oracle.py),
  1e-12;
* the Bloch-mode propagation constants of both gratings within 2e-9 of the
  reference's stored values (the 1D pencil is far from normal: eigenvalue
  errors run a few hundred times the Krylov residual of 1e-13), and the nodal
  values of the well-separated leading modes against the oracle's solve
  within 5e-5 of their largest value (up to a factor of modulus one per
  mode; the eigenvectors of clustered evanescent modes are less settled);
* end to end through the drop-in objects (NanoStruct('1D_array').calc_modes
  on the GPU, Stack.calc_scat): the reference's stored R_net, T_net within
  1e-6 (relative for the large entries of evanescent orders) and its txt
  spectra (R, T) within 1e-8.
"""
import os

import numpy as np
import pytest

from oracle import fem1d_oracle as F1

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
FX = np.load(os.path.join(GOLD, 'fem1d.npz'))
CASE4 = np.load(os.path.join(GOLD, 'case_4.npz'), allow_pickle=True)


def _mesh(i):
    p = 'g%d_' % i
    tab = FX[p + 'table_nod'].astype(np.int64).T
    x = FX[p + 'x_arr']
    tel = FX[p + 'type_el'].astype(np.int64).copy()
    tel[(tel == 2) & (np.abs(x[tab[:, 0] - 1] - 0.37) < 1e-9)] = 1
    return x, tab, tel


def test_1d_element_matrices_and_assembly_match_the_oracle():
    from emustack_b200.fem import FemMesh1D, FemModeSolver
    x, tab, tel = _mesh(1)
    m = FemMesh1D(x, tab, tel)
    topo = F1.Topology1D(x, tab)
    n_eff, k0, bx, by = FX['g1_n_effs'], 2 * np.pi / 1.05, 0.4, -0.3
    K, M = F1.element_matrices(topo, n_eff, tel, k0, bx, by)
    Kg, Mg = F1.assemble(topo, K, M)
    s = FemModeSolver(m)
    s.factor(n_eff, k0, [bx, by], shift=300.0)
    rows = np.repeat(np.arange(m.neq, dtype=np.int64), np.diff(m.d_row_ptr.cpu().numpy()))
    cols = np.array(m.d_col.cpu().numpy(), dtype=np.int64)
    kref = np.asarray(Kg.tocsr()[rows, cols]).ravel()
    mref = np.asarray(Mg.tocsr()[rows, cols]).ravel()
    np.testing.assert_allclose(s.K.cpu().numpy(), kref, rtol=0, atol=1e-12 * np.abs(kref).max())
    np.testing.assert_allclose(s.M.cpu().numpy(), mref, rtol=0, atol=1e-12 * np.abs(mref).max())


@pytest.mark.parametrize('i', [1, 2])
def test_1d_fem_solve_matches_the_reference_and_the_oracle(i):
    from emustack_b200.fem import FemMesh1D, FemModeSolver
    p = 'g%d_' % i
    x, tab, tel = _mesh(i)
    bloch = [float(FX[p + 'kx']), float(FX[p + 'ky'])]
    wln, nval = float(FX[p + 'wl_norm']), int(FX[p + 'num_BMs'])
    shift = complex(FX[p + 'shift']).real
    s = FemModeSolver(FemMesh1D(x, tab, tel))
    b1, s1, b2, s2 = s.solve_pair(FX[p + 'n_effs'], wln, bloch, nval, shift=shift)
    np.testing.assert_allclose(b1, CASE4['p0_lay%d_k_z' % i], rtol=2e-9, atol=0)
    ob1, os1, ob2, os2 = F1.solve_modes(x, tab, tel, FX[p + 'n_effs'], wln, bloch[0], bloch[1], nval, shift)
    np.testing.assert_allclose(b2, ob2, rtol=2e-9, atol=0)
    gap = np.minimum(np.r_[np.abs(np.diff(b1)), np.inf], np.r_[np.inf, np.abs(np.diff(b1))])
    sep = np.nonzero(gap[:16] > 1e-2 * np.abs(b1[:16]))[0]
    assert len(sep) >= 4
    # array_sol_1d.f divides each mode by its largest value on one half of
    # the cell; in these mirror-symmetric gratings the two halves hold equal
    # largest values up to rounding, so the two solves may pick mirror points
    # and differ by a factor of modulus one: compared up to that factor
    g1, g2 = s1.cpu().numpy(), s2.cpu().numpy()
    for k in sep:
        for got, ref in ((g1, os1), (g2, os2)):
            a, b = got[:, k].ravel(), ref[:, k].ravel()
            c = np.vdot(a, b) / np.vdot(a, a)
            assert abs(abs(c) - 1.0) < 1e-5, (k, c)
            np.testing.assert_allclose(c * a, b, rtol=0, atol=5e-5 * np.abs(b).max(), err_msg='mode %d' % k)


def test_drop_in_stack_of_gpu_gratings_matches_the_reference():
    from emustack_b200 import materials, objects
    from emustack_b200.mesh import Mesh1D
    from emustack_b200.stack import Stack
    period = 760.0
    light = objects.Light(800.0, max_order_PWs=6, theta=0.0, phi=0.0)
    sub = objects.ThinFilm(period, height_nm='semi_inf', world_1d=True, material=materials.Air, loss=False)
    sup = objects.ThinFilm(period, height_nm='semi_inf', world_1d=True, material=materials.Air, loss=False)
    lays = [sub.calc_modes(light)]
    for i, h in ((1, 150.0), (2, 900.0)):
        x, tab, tel = _mesh(i)
        n = FX['g%d_n_effs' % i]
        mats = dict(background=materials.Material(complex(n[0])), inclusion_a=materials.Material(complex(n[1])))
        if len(n) > 2:
            mats['inclusion_b'] = materials.Material(complex(n[2]))
        ns = objects.NanoStruct('1D_array', period, 190, height_nm=h, world_1d=True, loss=True,
                                mesh=Mesh1D(x, tab, tel), **mats)
        sim = ns.calc_modes(light)
        np.testing.assert_allclose(sim.k_z, CASE4['p0_lay%d_k_z' % i], rtol=2e-9)
        lays.append(sim)
    lays.append(sup.calc_modes(light))
    st = Stack(tuple(lays))
    st.calc_scat(pol='TE')
    np.testing.assert_allclose(np.asarray(st.R_net), CASE4['p0_R_net'], rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(np.asarray(st.T_net), CASE4['p0_T_net'], rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(float(np.real(st.r_list[0])), CASE4['txt_Reflectance_stack0001'][0][1], rtol=0,
                               atol=1e-8)
    np.testing.assert_allclose(float(np.real(st.t_list[-1])), CASE4['txt_Transmittance_stack0001'][0][1], rtol=0,
                               atol=1e-8)
    # x-z slices through the two gratings (fields_vertically's 1D branch)
    # against the restatement of its loop, from the same modes and amplitudes
    from emustack_b200.fields import fields_vertically
    from oracle import fields_oracle as FO
    import tempfile
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.chdir(tmp)
        try:
            res = fields_vertically([st])[0]
        finally:
            os.chdir(cwd)
    nl = len(st.layers)
    hn = st.heights_norm()
    for lay in (1, 2):
        layer = st.layers[lay]
        vi = nl - lay - 1
        vc = np.concatenate([np.asarray(st.vec_coef_down[vi]).ravel(), np.asarray(st.vec_coef_up[vi]).ravel()])
        z = np.linspace(0.0, hn[lay - 1], len(res['z_%d' % lay]))
        ref = FO.vertical_slice_1d(layer.sol1.cpu().numpy(), layer.k_z, vc, hn[lay - 1], z)
        for c, name in enumerate('xyz'):
            got = res['E_%s_%d' % (name, lay)]
            assert got.shape == (2 * len(_mesh(lay)[1]) + 1, len(z))
            np.testing.assert_allclose(got, ref[c], rtol=0, atol=1e-12 * max(np.abs(ref[c]).max(), 1e-300))
