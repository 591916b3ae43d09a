"""Host side of the FEM mode solve (emu_fem_topology, no GPU needed): the
periodic pairing, DOF numbering, edge orientation and CSR pattern against
the oracle's restatement of periodic_node.f / periodic_cond.f / basis_ls.f,
on the reference's own test meshes; and the CSR gather of element entries
reproducing the oracle's assembled K and M."""
import os

import numpy as np
import pytest

from emustack_b200.fem import FemMesh, mode_order
from oracle import fem_oracle as F
from oracle.overlap1d_oracle import z_indexx

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


@pytest.mark.parametrize('name', ['4testing-600_120.mail', '4testing-940_266_sq.mail'])
def test_topology_matches_the_oracle(name):
    path = os.path.join(GOLD, name)
    m = FemMesh.from_mail(path, device='cpu')
    x, tn, tab, tel = F.read_mail(path)
    topo = F.Topology(x, tn, tab)
    assert m.neq == topo.neq
    np.testing.assert_array_equal(m.dof, topo.dof)
    np.testing.assert_array_equal(m.ends, topo.ends)
    np.testing.assert_allclose(m.shift, topo.shift, rtol=0, atol=1e-12)
    # every boundary node has an image a lattice vector away: shifts are 0 or +-1
    assert set(np.unique(np.round(m.shift, 9))) <= {-1.0, 0.0, 1.0}


def test_csr_gather_reproduces_the_oracle_assembly():
    path = os.path.join(GOLD, '4testing-600_120.mail')
    m = FemMesh.from_mail(path, device='cpu')
    x, tn, tab, tel = F.read_mail(path)
    topo = F.Topology(x, tn, tab)
    K, M = F.element_matrices(topo, x, [1.0, 3.5 + 0.01j], tel, 2 * np.pi / 0.9, [0.3, -0.2])
    Kg, Mg = F.assemble(topo, K, M)
    sp, src = m.d_src_ptr.numpy(), m.d_src.numpy()
    rows = np.repeat(np.arange(m.neq, dtype=np.int64), np.diff(m.d_row_ptr.numpy()))
    cols = np.array(m.d_col.numpy(), dtype=np.int64)
    Kf, Mf = K.ravel(), M.ravel()
    Kc = np.add.reduceat(Kf[src], sp[:-1])
    Mc = np.add.reduceat(Mf[src], sp[:-1])
    Kd, Md = Kg.tocsr(), Mg.tocsr()
    np.testing.assert_allclose(Kc, np.asarray(Kd[rows, cols]).ravel(), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(Mc, np.asarray(Md[rows, cols]).ravel(), rtol=1e-12, atol=1e-12)
    Kd.eliminate_zeros()
    assert len(cols) >= Kd.nnz


def test_mode_order_is_the_reference_quicksort():
    rng = np.random.default_rng(3)
    beta = rng.normal(size=50) + 1j * rng.normal(size=50) * 0.1
    beta[7] = beta[3]          # a tie
    beta[20] = -beta[11]       # equal beta^2
    np.testing.assert_array_equal(mode_order(beta), z_indexx(-np.real(beta * beta)))


def test_topology_refuses_a_boundary_node_without_image():
    """A boundary node with no periodic partner is refused (periodic_node.f
    stops there), as are missing buffers and out-of-range node numbers."""
    import ctypes as C
    from emustack_b200 import _lib
    path = os.path.join(GOLD, '4testing-600_120.mail')
    x, tn, tab, tel = F.read_mail(path)
    x = x.copy()
    b = int(np.nonzero(tn)[0][0])
    x[b] += 0.01                      # breaks its pairing
    with pytest.raises(_lib.EmuError):
        FemMesh(x, tn, tab, tel, device='cpu')
    bad = tab.copy()
    bad[0, 0] = len(x) + 1
    with pytest.raises(_lib.EmuError):
        FemMesh(F.read_mail(path)[0], tn, bad, tel, device='cpu')
    t = _lib.EmuFemTopology()
    t.npt, t.nel = 3, 1
    assert _lib.lib().emu_fem_topology(C.byref(t)) == _lib.EMU_E_ARG


def test_fem_device_entries_check_arguments_on_the_host():
    """Shape and pointer checks of the device entry points return before any
    launch (no GPU needed)."""
    import ctypes as C
    from emustack_b200 import _lib
    L = _lib.lib()
    z = _lib.EmuC128(0.0, 0.0)
    assert L.emu_fem_lu(0, None, 1, None, None, None) == _lib.EMU_E_SHAPE
    assert L.emu_fem_lu(4, None, 4, None, None, None) == _lib.EMU_E_ARG
    assert L.emu_fem_inverse(4, None, 4, None, 5, None, None, 5, None) == _lib.EMU_E_SHAPE
    assert L.emu_fem_shifted_dense(4, None, None, None, None, z, None, 3, None) == _lib.EMU_E_SHAPE
    assert L.emu_fem_apply_op(4, 2, None, 4, 4, None, None, None, None, None, 2, None, None, 2, None) == \
        _lib.EMU_E_ARG
    assert L.emu_fem_assemble(-1, None, None, None, None, None, None, None) == _lib.EMU_E_SHAPE
    e = _lib.EmuFemElements()
    e.nel, e.n_types = 1, 9
    assert L.emu_fem_element_matrices(C.byref(e), None) == _lib.EMU_E_ARG
    f = _lib.EmuFemFields()
    f.nel, f.neq, f.nval, f.ldv = 1, 1, 2, 1
    assert L.emu_fem_nodal_fields(C.byref(f), None, 0, None) == _lib.EMU_E_ARG


def test_1d_topology_matches_the_oracle():
    """emu_fem1d_topology: the DOF numbering and periodic shifts of
    periodic_cond_1d.f as the oracle restates them, on the reference's own
    case-4 grating mesh; the CSR gather reproduces the oracle's assembly;
    unordered elements are refused."""
    from emustack_b200 import _lib
    from emustack_b200.fem import FemMesh1D
    from oracle import fem1d_oracle as F1
    d = np.load(os.path.join(GOLD, 'fem1d.npz'))
    tab = d['g1_table_nod'].astype(np.int64).T
    x, tel = d['g1_x_arr'], d['g1_type_el'].astype(np.int64)
    m = FemMesh1D(x, tab, tel, device='cpu')
    topo = F1.Topology1D(x, tab)
    assert m.neq == topo.neq == 9 * len(tab)
    np.testing.assert_array_equal(m.dof, topo.dof)
    np.testing.assert_allclose(m.shift, topo.shift, rtol=0, atol=1e-15)
    K, M = F1.element_matrices(topo, d['g1_n_effs'], tel, 2 * np.pi / 1.05, 0.3, -0.2)
    Kg, Mg = F1.assemble(topo, K, M)
    sp, src = m.d_src_ptr.numpy(), m.d_src.numpy()
    rows = np.repeat(np.arange(m.neq, dtype=np.int64), np.diff(m.d_row_ptr.numpy()))
    cols = np.array(m.d_col.numpy(), dtype=np.int64)
    Kc = np.add.reduceat(K.ravel()[src], sp[:-1])
    Mc = np.add.reduceat(M.ravel()[src], sp[:-1])
    np.testing.assert_allclose(Kc, np.asarray(Kg.tocsr()[rows, cols]).ravel(), rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(Mc, np.asarray(Mg.tocsr()[rows, cols]).ravel(), rtol=1e-13, atol=1e-13)
    with pytest.raises(_lib.EmuError):
        FemMesh1D(x, tab[::-1].copy(), tel, device='cpu')
