"""The FEM oracle (oracle/fem_oracle.py) against the reference's stored
results for its own test cases 1 and 2 (the mesh 4testing-600_120.mail): the
Bloch-mode propagation constants the reference's FEM found, and, through the
overlap and GSM oracles, the layer's interface reflection R12, the stack's
R_net / T_net and the absorptance / transmittance / reflectance lists.

Quantities that depend on each mode's normalisation (T12, R21, T21) are
checked up to one complex factor per mode: the reference's stored matrices
and the oracle's agree row by row (T12) within that factor for every mode
whose eigenvalue is separated from its neighbours; the reference's own test
of these matrices is disabled (tests/test_case_1_simple_struct.py:131-148).
The inputs of the solve (indices, Bloch vector, shift) are the reference's,
recorded by tests/golden/make_fem_golden.py."""
import os

import numpy as np
import pytest

from oracle import fem_oracle as F
from oracle import gsm_oracle as G
from oracle import overlap as OV

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, 'golden')


def _mesh():
    return F.read_mail(os.path.join(GOLD, '4testing-600_120.mail'))


def solve_case(case, p):
    """Modes, J, J_dag and the stack of one golden point through the oracles."""
    fem = np.load(os.path.join(GOLD, 'fem.npz'))
    gold = np.load(os.path.join(GOLD, case.replace('case', 'case_') + '.npz'), allow_pickle=True)
    key = '%s_p%d_' % (case, p)
    x, tn, tab, tel = _mesh()
    wl_norm = float(fem[key + 'wl_norm'])
    bloch = np.asarray(fem[key + 'k_pll_norm'], float)
    nval = int(fem[key + 'num_BMs'])
    mo = int(fem[key + 'max_order'])
    b1, s1, b2, s2 = F.solve_modes(x, tn, tab, tel, fem[key + 'n_effs'], wl_norm, bloch, nval,
                                   shift=complex(fem[key + 'shift']).real)
    k0 = 2 * np.pi / wl_norm
    ovl, perm, scale, warn, s2n, b2n = OV.orthogonal_normalise(x, tab, tel, np.ones(2, complex), b1, b2,
                                                              s1, s2, k0)
    inv, px, py = OV.pw_ordering(mo, 1.0, 1.0, bloch, k0)
    J = OV.J_overlap(x, tab, s1, 1.0, 1.0, bloch, inv, mo)
    Jd = OV.J_dagger_overlap(x, tab, s2n, 1.0, 1.0, bloch, inv, mo)
    g = 'p%d_' % p
    wl, kp, per = float(gold[g + 'wl_nm']), gold[g + 'k_pll'], float(gold[g + 'period'])
    air = G.make_air_ref(wl, kp, per, per, mo)
    sub = G.film_layer(gold[g + 'lay0_n'], wl, kp, per, air, None, per, mo, loss=bool(gold[g + 'lay0_loss']))
    sup = G.film_layer(gold[g + 'lay2_n'], wl, kp, per, air, None, per, mo, loss=bool(gold[g + 'lay2_loss']))
    ns = G.OracleLayer('struct', b1, height_nm=float(gold[g + 'heights_nm'][0]), J=J, J_dag=Jd)
    out = G.calc_scat([sub, ns, sup], air, per, pol=str(gold[g + 'pol']))
    return b1, out, gold, g


@pytest.mark.parametrize('case,p', [('case1', 0), ('case2', 0)])
def test_fem_oracle_matches_the_reference(case, p):
    b1, out, gold, g = solve_case(case, p)
    ref_kz = gold[g + 'lay1_k_z']
    np.testing.assert_allclose(b1, ref_kz, rtol=1e-10, atol=0)
    R12, T12, R21, T21 = out.interfaces[1]
    np.testing.assert_allclose(R12, gold[g + 'lay1_R12'], rtol=0, atol=1e-6)
    for k in ('R_net', 'T_net'):
        np.testing.assert_allclose(getattr(out, k), gold[g + k], rtol=0, atol=1e-6)
    for k in ('a_list', 't_list', 'r_list'):
        np.testing.assert_allclose(np.asarray(getattr(out, k), float), gold[g + k], rtol=1e-6, atol=1e-7)
    # T12 rows of separated modes: one complex factor per mode
    ref = gold[g + 'lay1_T12']
    gap = np.minimum(np.r_[np.abs(np.diff(b1)), np.inf], np.r_[np.inf, np.abs(np.diff(b1))])
    checked = 0
    for i in np.nonzero(gap > 1e-3 * np.abs(b1))[0]:
        big = np.abs(ref[i]) > 1e-3 * np.abs(ref[i]).max()
        r = T12[i, big] / ref[i, big]
        assert np.abs(r - r[0]).max() < 1e-5 * abs(r[0]), i
        checked += 1
    assert checked >= 4


def test_fem_oracle_on_the_gold_hole_mesh_matches_the_reference_case_5():
    """The oracle's prime solve on the reference's second test mesh
    (4testing-940_266_sq.mail: 266 nm square holes in gold at period 940 nm,
    30 336 DOFs) with the inputs the reference passes for its test case 5
    (100 Bloch modes, 1043.4 nm, 5 degrees) against its stored k_z."""
    fem = np.load(os.path.join(GOLD, 'fem.npz'))
    key = 'case5_p0_'
    ref = np.load(os.path.join(GOLD, 'case_5.npz'), allow_pickle=True)['p0_lay1_k_z']
    x, tn, tab, tel = F.read_mail(os.path.join(GOLD, '4testing-940_266_sq.mail'))
    topo = F.Topology(x, tn, tab)
    k0 = 2 * np.pi / float(fem[key + 'wl_norm'])
    bloch = np.asarray(fem[key + 'k_pll_norm'], float)
    K, M = F.element_matrices(topo, x, fem[key + 'n_effs'], tel, k0, bloch)
    Kg, Mg = F.assemble(topo, K, M)
    b2, _ = F.eigen_solve(Kg, Mg, int(fem[key + 'num_BMs']), complex(fem[key + 'shift']).real)
    beta = F.beta_from(b2)
    beta = beta[F.z_indexx(-np.real(beta ** 2))]
    np.testing.assert_allclose(beta, ref, rtol=1e-9, atol=0)
