"""Generate tests/golden/fem1d.npz: what the EMUstack reference passes to its
1D FEM mode solver (calc_modes_1d, backend/mode_calcs.py:331-341) for the two
gratings of its test case 4 (tests/test_case_4_stacked_gratings.py: period
760 nm, 800 nm light, max order 6, world_1d): the 1D mesh its NanoStruct built
(P2 node coordinates, element table, material types), the materials' indices,
the normalised Bloch vector, the shift and the number of Bloch modes.  The
reference's Simmo.calc_modes runs up to the Fortran call, which is
intercepted here.  The reference's results for these layers (k_z, interface
and net matrices) are in case_4.npz.

    EMUSTACK_REF=<path to the EMUstack tree> python tests/golden/make_fem1d_golden.py
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
    names = ('wl_norm', 'num_BMs', 'max_order', 'nb_typ_el', 'n_msh_pts', 'n_msh_el', 'table_nod', 'type_el',
             'x_arr', 'itermax', 'debug', 'mesh_file', 'n_effs', 'kx', 'ky', 'shift')

    def capture(*args):
        seen.update(zip(names, args))
        seen['world_1d'] = args[-1]
        seen['num_pw_per_pol'] = args[-3]
        raise _Captured()

    fortran.calc_modes_1d = capture
    # the 1D NanoStruct draws its mesh when it builds it: a permissive stand-in
    # for the plotting calls (the image is not needed)
    class _Any(object):
        def __getattr__(self, name):
            return _Any()

        def __call__(self, *a, **k):
            return _Any()

        def __iter__(self):
            return iter((_Any(), _Any()))

    sys.modules['matplotlib.pyplot'].__getattr__ = lambda name: _Any()
    objects.plt = _Any() if hasattr(objects, 'plt') else getattr(objects, 'plt', None)
    period = 760
    light = objects.Light(800.0, max_order_PWs=6, theta=0.0, phi=0.0)
    g1 = objects.NanoStruct('1D_array', period, diameter1=int(round(0.25 * period)),
                            diameter2=int(round(0.25 * period)), height_nm=150,
                            inclusion_a=materials.Material(1.46 + 0.0j), inclusion_b=materials.Material(1.46 + 0.0j),
                            background=materials.Material(3.61 + 0.0j), loss=True, lc_bkg=0.005)
    g2 = objects.NanoStruct('1D_array', period, int(round(0.25 * period)), height_nm=900,
                            background=materials.Material(3.61 + 0.0j), inclusion_a=materials.Material(1.46 + 0.0j),
                            loss=True, lc_bkg=0.005)
    d = {}
    for i, g in enumerate((g1, g2)):
        seen.clear()
        try:
            g.calc_modes(light)
        except _Captured:
            pass
        for k in ('wl_norm', 'num_BMs', 'max_order', 'nb_typ_el', 'table_nod', 'type_el', 'x_arr', 'n_effs',
                  'kx', 'ky', 'shift', 'world_1d', 'num_pw_per_pol'):
            d['g%d_%s' % (i + 1, k)] = np.asarray(seen[k])
    out = os.path.join(HERE, 'fem1d.npz')
    np.savez_compressed(out, **d)
    print('wrote', out, sorted(d))


if __name__ == '__main__':
    main()
