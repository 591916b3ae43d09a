"""Generate tests/golden/fem.npz: the arguments the EMUstack reference passes to
its FEM mode solver (calc_modes_2d, backend/mode_calcs.py:371-381) for the
nanostructured layer of its test cases 1 and 2 (tests/test_case_1_simple_struct.py,
tests/test_case_2_simple_non_norm_inc.py: the mesh 4testing-600_120.mail, a
120 nm Si_c wire in air at period 600 nm) and of its test case 5
(tests/test_case_5_EOT_5_degrees.py.bak: the mesh 4testing-940_266_sq.mail,
266 nm square holes in gold at period 940 nm, 100 Bloch modes, 5 degrees).  The reference's Simmo.calc_modes
runs up to the Fortran call, which is intercepted here and its inputs
recorded: normalised wavelength, number of Bloch modes, plane-wave order,
the materials' indices (loss applied), the normalised Bloch vector and the
shift of the shift-and-invert solve.  The reference's results for these
layers (k_z, interface and net matrices) are in case_1.npz, case_2.npz and
case_5.npz.

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
    wire = dict(period=600, diameter=120, height_nm=2330, inclusion_a=materials.Si_c, background=materials.Air,
                mesh_file='4testing-600_120.mail')
    holes = dict(period=940, diameter=266, height_nm=200, inclusion_a=materials.Air, background=materials.Au,
                 inc_shape='square', mesh_file='4testing-940_266_sq.mail')
    cases = {'case1': ([500.0, 1000.0], 2, 0.0, 0.0, 40, wire), 'case2': ([500.0], 1, 20.0, 40.0, 20, wire),
             'case5': ([1.11 * 940], 4, 5.0, 0.0, 100, holes)}
    d = {}
    for name, (wls, max_order, theta, phi, num_BMs, geo) in cases.items():
        for i, wl in enumerate(wls):
            light = objects.Light(wl, max_order_PWs=max_order, theta=theta, phi=phi)
            g = dict(geo)
            ns = objects.NanoStruct('2D_array', g.pop('period'), g.pop('diameter'), loss=True, make_mesh_now=False,
                                    **g)
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
