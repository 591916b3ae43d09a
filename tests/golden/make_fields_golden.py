"""Generate tests/golden/fields.npz from the EMUstack reference: the
reference's own ``field_values`` (backend/plotting.py:2857-2996) and
``t_r_a_write_files`` (backend/plotting.py:735-809) run on stacks that the
reference's GSM solved.

    EMUSTACK_REF=<path to the EMUstack tree> python tests/golden/make_fields_golden.py

The reference is imported as tests/golden/make_golden.py imports it, with two
more shims for running its Python-2 era plotting module under Python 3:
``xrange = range`` and ``scipy.sqrt`` (removed from scipy) set to numpy's
``emath.sqrt``, the function it used to be.  The files the reference writes
go to a scratch directory (``EMUSTACK_SCRATCH``, default ``_work/fields_golden``
under the repository root); their contents are stored in the fixture.
"""
from __future__ import annotations

import builtins
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)


def main():
    import make_golden
    objects, materials, stack, mode_calcs = make_golden.import_reference()
    builtins.xrange = range
    import scipy
    if not hasattr(scipy, 'sqrt'):
        scipy.sqrt = np.emath.sqrt
    import plotting

    scratch = os.environ.get('EMUSTACK_SCRATCH', os.path.join(ROOT, '_work', 'fields_golden'))
    os.makedirs(scratch, exist_ok=True)

    d = {}
    # (name, period, world_1d, max_order, theta, phi, pol, wavelengths, layers bottom to top)
    # layer: (n, height_nm or 'semi_inf', loss)
    specs = [
        ('s2d', 500.0, False, 2, 20.0, 30.0, 'TM', [450.0, 700.0],
         [(1.46, 'semi_inf', False), (3.6 + 0.27j, 80, True), (2.0 + 0.01j, 150, True),
          (1.0, 'semi_inf', False)]),
        ('s2c', 450.0, False, 1, 35.0, 10.0, 'R Circ', [620.0],
         [(1.5, 'semi_inf', False), (2.4 + 0.05j, 60, True), (1.33, 'semi_inf', False)]),
        ('s1d', 600.0, True, 3, 15.0, 0.0, 'TE', [550.0],
         [(1.5, 'semi_inf', False), (2.5 + 0.1j, 120, True), (1.0, 'semi_inf', False)]),
    ]
    rng = np.random.default_rng(20261204)
    names = []
    for name, per, w1d, mo, th, ph, pol, wls, lays in specs:
        films = [objects.ThinFilm(period=per, height_nm=h, world_1d=w1d,
                                  material=materials.Material(n), loss=loss) for n, h, loss in lays]
        stacks = []
        for p, wl in enumerate(wls):
            key = '%s_p%d_' % (name, p)
            names.append(key)
            light = objects.Light(wl, max_order_PWs=mo, theta=th, phi=ph)
            sims = [f.calc_modes(light) for f in films]
            st = stack.Stack(sims)
            st.calc_scat(pol=pol)
            stacks.append(st)
            d[key + 'wl_nm'] = np.array(wl)
            d[key + 'theta_phi'] = np.array([th, ph])
            d[key + 'k_pll'] = np.asarray(light.k_pll, float)
            d[key + 'period'] = np.array(per)
            d[key + 'world_1d'] = np.array(w1d)
            d[key + 'max_order'] = np.array(mo)
            d[key + 'pol'] = np.array(pol)
            d[key + 'n'] = np.array([complex(n) for n, _, _ in lays])
            d[key + 'loss'] = np.array([loss for _, _, loss in lays])
            d[key + 'heights_nm'] = np.array([h for _, h, _ in lays[1:-1]], float)
            d[key + 'a_list'] = np.array([float(np.real(np.asarray(a)).ravel()[0]) for a in st.a_list])
            d[key + 't_list'] = np.array([float(np.real(np.asarray(a)).ravel()[0]) for a in st.t_list])
            d[key + 'r_list'] = np.array([float(np.real(np.asarray(a)).ravel()[0]) for a in st.r_list])
            d[key + 'vec_coef_down'] = np.array([np.asarray(v).ravel() for v in st.vec_coef_down])
            d[key + 'vec_coef_up'] = np.array([np.asarray(v).ravel() for v in st.vec_coef_up])
            os.chdir(scratch)
            for i, lay in enumerate(sims):
                lk = key + 'lay%d_' % i
                d[lk + 'alphas'] = np.asarray(lay.alphas, float)
                d[lk + 'betas'] = np.atleast_1d(np.asarray(lay.betas, float))
                d[lk + 'sort_order'] = np.asarray(lay.sort_order)
                d[lk + 'kz'] = np.asarray(lay.calc_kz())
                d[lk + 'n'] = np.array(complex(lay.n()))
                h = lay.structure.height_nm
                zmax = 0.5 if h == 'semi_inf' else float(h) / per
                pts = np.column_stack([rng.uniform(0, 1, 9), rng.uniform(0, 1, 9),
                                       np.concatenate([[0.0, zmax], rng.uniform(0, zmax, 7)])])
                d[lk + 'xyz'] = pts
                sp = plotting.field_values([st], lay_interest=i, xyz_values=[tuple(q) for q in pts])
                Ex, Ey, Ez, Et = (np.asarray(a) for a in sp[0])
                d[lk + 'E'] = np.array([Ex, Ey, Ez])
                d[lk + 'E_tot'] = np.asarray(Et)
        # the reference's text writer on this list of stacks
        os.chdir(scratch)
        for fn in os.listdir('.'):
            if fn.endswith('.txt'):
                os.remove(fn)
        plotting.t_r_a_write_files(stacks, np.array(wls), stack_label=7)
        txt = sorted(fn for fn in os.listdir('.') if fn.endswith('.txt'))
        d[name + '_txt_names'] = np.array(txt)
        d[name + '_txt_text'] = np.array([open(fn).read() for fn in txt])
    d['names'] = np.array(names)
    out = os.path.join(HERE, 'fields.npz')
    np.savez_compressed(out, **d)
    print('wrote', out, os.path.getsize(out), 'bytes')


if __name__ == '__main__':
    main()
