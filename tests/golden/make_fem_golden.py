"""Generate tests/golden/fem.npz: the arguments the EMUstack reference passes to
its FEM mode solver (calc_modes_2d, backend/mode_calcs.py:371-381) for the
nanostructured layer of its test cases 1 and 2 (tests/test_case_1_simple_struct.py,
tests/test_case_2_simple_non_norm_inc.py: the mesh 4testing-600_120.mail, a
120 nm Si_c wire in air at period 600 nm).  The reference's Simmo.calc_modes
runs up to the Fortran call, which is intercepted here and its inputs
recorded: normalised wavelength, number of Bloch modes, plane-wave order,
the materials' indices (loss applied), the normalised Bloch vector and the
shift of the shift-and-invert solve.  The reference's results for these
layers (k_z, interface and net matrices) are in case_1.npz / case_2.npz.

    EMUSTACK_REF=<path to the EMUstack tree> python tests/golden/make_fem_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)


class _Captured(Exception):
    pass


def main():
    import make_golden
    objects, materials, stack, mode_calcs = make_golden.import_reference()
    fortran = sys.modules['fortran.EMUstack']
    seen = {}

    def capture(*args):
        (seen['wl_norm'], seen['num_BMs'], seen['max_order'], _dbg, _path, seen['mesh_file'],
         seen['n_msh_pts'], seen['n_msh_el'], seen['nb_typ_el'], seen['n_effs'], seen['k_pll_norm'],
         seen['shift'], seen['E_H_field'], seen['i_cond'], seen['itermax']) = args[:15]
        raise _Captured()

    fortran.calc_modes_2d = capture
    cases = {'case1': ([500.0, 1000.0], 2, 0.0, 0.0, 40), 'case2': ([500.0], 1, 20.0, 40.0, 20)}
    d = {}
    for name, (wls, max_order, theta, phi, num_BMs) in cases.items():
        for i, wl in enumerate(wls):
            light = objects.Light(wl, max_order_PWs=max_order, theta=theta, phi=phi)
            ns = objects.NanoStruct('2D_array', 600, 120, height_nm=2330, inclusion_a=materials.Si_c,
                                    background=materials.Air, loss=True, make_mesh_now=False,
                                    mesh_file='4testing-600_120.mail')
            seen.clear()
            try:
                ns.calc_modes(light, num_BMs=num_BMs)
            except _Captured:
                pass
            key = '%s_p%d_' % (name, i)
            for k in ('wl_norm', 'num_BMs', 'max_order', 'n_effs', 'k_pll_norm', 'shift', 'E_H_field',
                      'i_cond', 'nb_typ_el', 'n_msh_pts', 'n_msh_el'):
                d[key + k] = np.asarray(seen[k])
            d[key + 'mesh_file'] = np.asarray(str(seen['mesh_file']))
    out = os.path.join(HERE, 'fem.npz')
    np.savez_compressed(out, **d)
    print('wrote', out, len(d), 'arrays')


if __name__ == '__main__':
    main()
