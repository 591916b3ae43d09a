"""GPU parity of the FEM Bloch-mode solve (emustack_b200.fem, csrc/fem.cu).

* Element matrices and the assembled K, M against the oracle's restatement
  of asmbly.f (oracle/fem_oracle.py), 1e-12.
* The full solve on the reference's own test mesh (4testing-600_120.mail)
  with the inputs the reference passes (tests/golden/fem.npz): the Bloch-mode
  propagation constants of the reference's stored cases 1 and 2 within 1e-10
  relative; the nodal fields of every well-separated mode against the
  oracle's solve, 5e-6 of the mode's largest value (both solves converge
  their eigenvectors to about 1e-14 / gap).
* End to end through the drop-in objects (NanoStruct.calc_modes on the GPU,
  Stack.calc_scat): the reference's stored R12 of the layer, R_net, T_net
  and a/t/r lists within 1e-6 (the reference's own test tolerance).
* A second, larger mesh: the gold film with square holes of the reference's
  test case 5 (4testing-940_266_sq.mail, 2 528 elements, 30 336 DOFs, 100
  Bloch modes at 5 degrees), its stored propagation constants within 1e-9.
"""
import os

import numpy as np
import pytest
import torch

from oracle import fem_oracle as F

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, 'golden')
MAIL = os.path.join(GOLD, '4testing-600_120.mail')
FEM = np.load(os.path.join(GOLD, 'fem.npz'))


def _case(case, p):
    key = '%s_p%d_' % (case, p)
    gold = np.load(os.path.join(GOLD, case.replace('case', 'case_') + '.npz'), allow_pickle=True)
    return key, gold, 'p%d_' % p


def test_element_matrices_and_assembly_match_the_oracle():
    from emustack_b200.fem import FemMesh, FemModeSolver
    m = FemMesh.from_mail(MAIL)
    x, tn, tab, tel = F.read_mail(MAIL)
    topo = F.Topology(x, tn, tab)
    n_eff, k0, bloch = [1.0, 4.293 + 0.045j], 2 * np.pi / 0.83, [0.4, -0.7]
    K, M = F.element_matrices(topo, x, n_eff, tel, k0, bloch)
    s = FemModeSolver(m)
    s.factor(n_eff, k0, bloch, shift=1000.0)
    Kg, Mg = F.assemble(topo, K, M)
    rows = np.repeat(np.arange(m.neq, dtype=np.int64), np.diff(m.d_row_ptr.cpu().numpy()))
    cols = np.array(m.d_col.cpu().numpy(), dtype=np.int64)
    Kd, Md = Kg.tocsr(), Mg.tocsr()
    kref = np.asarray(Kd[rows, cols]).ravel()
    mref = np.asarray(Md[rows, cols]).ravel()
    np.testing.assert_allclose(s.K.cpu().numpy(), kref, rtol=0, atol=1e-12 * np.abs(kref).max())
    np.testing.assert_allclose(s.M.cpu().numpy(), mref, rtol=0, atol=1e-12 * np.abs(mref).max())


@pytest.mark.parametrize('case,p', [('case1', 0), ('case1', 1), ('case2', 0)])
def test_fem_solve_matches_the_reference_and_the_oracle(case, p):
    from emustack_b200.fem import FemMesh, FemModeSolver
    key, gold, g = _case(case, p)
    m = FemMesh.from_mail(MAIL)
    s = FemModeSolver(m)
    nval = int(FEM[key + 'num_BMs'])
    wl_norm = float(FEM[key + 'wl_norm'])
    bloch = np.asarray(FEM[key + 'k_pll_norm'], float)
    shift = complex(FEM[key + 'shift']).real
    b1, s1 = s.solve(FEM[key + 'n_effs'], wl_norm, bloch, nval, shift=shift)
    ref = gold[g + 'lay1_k_z']
    np.testing.assert_allclose(b1, ref, rtol=1e-10, atol=0)
    # nodal fields of separated modes against the oracle's solve
    x, tn, tab, tel = F.read_mail(MAIL)
    topo = F.Topology(x, tn, tab)
    K, M = F.element_matrices(topo, x, FEM[key + 'n_effs'], tel, 2 * np.pi / wl_norm, bloch)
    Kg, Mg = F.assemble(topo, K, M)
    b2, vec = F.eigen_solve(Kg, Mg, nval, shift)
    bo = F.beta_from(b2)
    order = F.z_indexx(-np.real(bo ** 2))
    so = F.nodal_fields(topo, vec[:, order], bloch)
    sg = s1.cpu().numpy()
    gap = np.minimum(np.r_[np.abs(np.diff(b1)), np.inf], np.r_[np.inf, np.abs(np.diff(b1))])
    sep = np.nonzero(gap > 1e-3 * np.abs(b1))[0]
    assert len(sep) >= 4
    for i in sep:
        scale = np.abs(so[:, i]).max()
        np.testing.assert_allclose(sg[:, i], so[:, i], rtol=0, atol=5e-6 * scale, err_msg='mode %d' % i)


@pytest.mark.parametrize('case,p,theta,phi', [('case1', 0, 0.0, 0.0), ('case2', 0, 20.0, 40.0)])
def test_drop_in_stack_with_gpu_modes_matches_the_reference(case, p, theta, phi):
    from emustack_b200 import materials, objects
    from emustack_b200.mesh import Mesh
    from emustack_b200.stack import Stack
    key, gold, g = _case(case, p)
    per = float(gold[g + 'period'])
    light = objects.Light(float(gold[g + 'wl_nm']), max_order_PWs=int(FEM[key + 'max_order']),
                          theta=theta, phi=phi)
    np.testing.assert_allclose(np.asarray(light.k_pll) * per, FEM[key + 'k_pll_norm'], rtol=1e-12, atol=1e-18)
    n_effs = FEM[key + 'n_effs']
    ns = objects.NanoStruct('2D_array', per, 120, height_nm=float(gold[g + 'heights_nm'][0]),
                            background=materials.Material(complex(n_effs[0])),
                            inclusion_a=materials.Material(complex(n_effs[1])), loss=True,
                            mesh=Mesh.from_mail(MAIL))
    sub = objects.ThinFilm(period=per, height_nm='semi_inf', material=materials.Material(complex(gold[g + 'lay0_n'])),
                           loss=bool(gold[g + 'lay0_loss']))
    sup = objects.ThinFilm(period=per, height_nm='semi_inf', material=materials.Material(complex(gold[g + 'lay2_n'])),
                           loss=bool(gold[g + 'lay2_loss']))
    sim = ns.calc_modes(light, num_BMs=int(FEM[key + 'num_BMs']))
    np.testing.assert_allclose(sim.k_z, gold[g + 'lay1_k_z'], rtol=1e-10)
    st = Stack((sub.calc_modes(light), sim, sup.calc_modes(light)))
    st.calc_scat(pol=str(gold[g + 'pol']))
    np.testing.assert_allclose(np.asarray(st.layers[1].R12), gold[g + 'lay1_R12'], rtol=0, atol=1e-6)
    np.testing.assert_allclose(np.asarray(st.R_net), gold[g + 'R_net'], rtol=0, atol=1e-6)
    np.testing.assert_allclose(np.asarray(st.T_net), gold[g + 'T_net'], rtol=0, atol=1e-6)
    for k in ('a_list', 't_list', 'r_list'):
        np.testing.assert_allclose(np.asarray(getattr(st, k), float), gold[g + k], rtol=1e-6, atol=1e-7)


def test_tensor_core_J_meets_the_bar_on_physical_modes():
    """J / J_dag of the GPU FEM modes of the reference's test layer (case 1,
    500 nm) by the split-TF32 x3 tensor-core contraction give the same a/t/r
    lists as the FP64 contraction within 1e-6 through the drop-in Stack (on
    random synthetic fields the same contraction is not held to that bar)."""
    from emustack_b200 import materials, objects
    from emustack_b200.fem import FemMesh, FemModeSolver
    from emustack_b200.mesh import Mesh
    from emustack_b200.stack import Stack
    key, gold, g = _case('case1', 0)
    fs = FemModeSolver(FemMesh.from_mail(MAIL))
    b1, s1, b2, s2 = fs.solve_pair(FEM[key + 'n_effs'], float(FEM[key + 'wl_norm']), FEM[key + 'k_pll_norm'],
                                   int(FEM[key + 'num_BMs']), shift=complex(FEM[key + 'shift']).real)
    per = float(gold[g + 'period'])
    light = objects.Light(float(gold[g + 'wl_nm']), max_order_PWs=int(FEM[key + 'max_order']), theta=0.0, phi=0.0)
    mesh = Mesh.from_mail(MAIL)
    n_effs = FEM[key + 'n_effs']
    ns = objects.NanoStruct('2D_array', per, 120, height_nm=float(gold[g + 'heights_nm'][0]),
                            background=materials.Material(complex(n_effs[0])),
                            inclusion_a=materials.Material(complex(n_effs[1])), loss=True, mesh=mesh)
    films = [objects.ThinFilm(period=per, height_nm='semi_inf', material=materials.Material(complex(gold[k])),
                              loss=False) for k in (g + 'lay0_n', g + 'lay2_n')]
    lists = {}
    for prec in ('fp64', 'tf32x3'):
        sim = ns.calc_modes(light, k_z=b1, fields={'sol1': s1, 'sol2': s2, 'beta1': b1, 'mesh': mesh,
                                                    'precision': prec})
        st = Stack((films[0].calc_modes(light), sim, films[1].calc_modes(light)))
        st.calc_scat(pol='TE')
        lists[prec] = np.concatenate([np.ravel(np.asarray(v, dtype=complex)).real
                                      for lst in (st.a_list, st.t_list, st.r_list) for v in lst])
    np.testing.assert_allclose(lists['tf32x3'], lists['fp64'], rtol=0, atol=1e-6)


def test_sweep_of_solves_equals_one_by_one():
    """fem.solve_pairs (several host threads and streams) returns what the
    solves give one after the other, within the solves' own accuracy (1e-10,
    the tolerance of the parity tests above; cuBLAS's reductions in the
    Krylov basis may round differently when several streams run at once)."""
    from emustack_b200.fem import FemMesh, FemModeSolver, solve_pairs
    m = FemMesh.from_mail(MAIL)
    key = 'case1_p0_'
    n_effs = FEM[key + 'n_effs']
    jobs = [(n_effs, w, np.asarray(FEM[key + 'k_pll_norm'], float) * (1.0 + 0.1 * i), None)
            for i, w in enumerate((0.8, 0.9, 1.1))]
    got = solve_pairs(m, jobs, 24, workers=3)
    s = FemModeSolver(m)
    for job, g in zip(jobs, got):
        ref = s.solve_pair(job[0], job[1], job[2], 24, concurrent=False)
        np.testing.assert_allclose(g[0], ref[0], rtol=1e-10, atol=0)
        np.testing.assert_allclose(g[2], ref[2], rtol=1e-10, atol=0)


def test_fem_solve_on_the_gold_hole_mesh_matches_the_reference_case_5():
    from emustack_b200.fem import FemMesh, FemModeSolver
    key = 'case5_p0_'
    ref = np.load(os.path.join(GOLD, 'case_5.npz'), allow_pickle=True)['p0_lay1_k_z']
    mesh = FemMesh.from_mail(os.path.join(GOLD, '4testing-940_266_sq.mail'))
    assert mesh.neq == 30336
    s = FemModeSolver(mesh)
    beta, sol = s.solve(FEM[key + 'n_effs'], float(FEM[key + 'wl_norm']), np.asarray(FEM[key + 'k_pll_norm'], float),
                        int(FEM[key + 'num_BMs']), shift=complex(FEM[key + 'shift']).real)
    np.testing.assert_allclose(beta, ref, rtol=1e-9, atol=0)
    assert np.all(np.isfinite(sol.cpu().numpy()))
    del s, sol
    torch.cuda.empty_cache()
