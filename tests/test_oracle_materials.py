"""The materials oracle (oracle.gsm_oracle.material_n) against the
reference's own Material.n (backend/materials.py:131-161) on constant,
tabulated (real and complex) and Drude materials: tests/golden/materials.npz,
made by tests/golden/make_materials_golden.py.  Bit for bit."""
import os

import numpy as np
import pytest

from oracle import gsm_oracle as G

GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'materials.npz'))


@pytest.mark.parametrize('name', ['const', 'complex_tab', 'real_tab', 'drude'])
@pytest.mark.parametrize('loss', [True, False])
def test_material_oracle_is_the_reference(name, loss):
    spec = GOLD['spec_' + name]
    spec = spec.item() if spec.shape == () else spec
    ref = GOLD['n_' + name] if loss else GOLD['n_' + name].real.astype(complex)
    got = np.array([complex(G.material_n(spec, w, loss)) for w in GOLD['wl']])
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize('name', ['const', 'complex_tab', 'real_tab', 'drude'])
def test_host_material_is_the_reference(name):
    """emustack_b200.materials.Material.n (the drop-in objects' host index)
    returns the reference's values bit for bit."""
    from emustack_b200.materials import Material
    spec = GOLD['spec_' + name]
    m = Material(spec.item() if spec.shape == () else spec)
    got = np.array([complex(np.asarray(m.n(w)).item()) for w in GOLD['wl']])
    np.testing.assert_array_equal(got, GOLD['n_' + name])
