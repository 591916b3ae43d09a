"""Generate the golden fixtures under tests/golden/ from the EMUstack reference.

Run where the reference source tree is available, with ``EMUSTACK_REF``
naming its root directory:

    EMUSTACK_REF=<path to the EMUstack tree> python tests/golden/make_golden.py

It imports the reference's own Python GSM (backend/stack.py,
backend/mode_calcs.py, backend/objects.py, backend/materials.py) with three
shims: ``np.mat = np.asmatrix`` (numpy 2 removed ``np.mat``), a stub
``fortran.EMUstack`` module (the FEM extension is not needed by the GSM
stage) and a stub ``matplotlib``.  Nanostructured layers cannot be
FEM-solved here, so:

* golden cases 1-5 are REPLAYED: each ``Simmo`` layer's interface matrices
  and Bloch-mode k_z are taken from the reference's stored
  tests/ref/case_N.npz and injected into the reference's interface memo
  (backend/mode_calcs.py:423-447) before ``Stack.calc_scat`` runs;
* synthetic nanostructured layers get seeded random J / J_dag (and k_z) and
  run through the reference's own ``r_t_mat_tf_ns``.

Each fixture stores the inputs needed to rerun the case without the reference
and the reference's outputs.  The files travel with the repository; nothing
at test time reads the reference tree.
"""
from __future__ import annotations

import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get('EMUSTACK_REF')


def import_reference():
    if not REF or not os.path.isdir(os.path.join(REF, 'backend')):
        raise SystemExit('set EMUSTACK_REF to the root of the EMUstack source tree')
    if not hasattr(np, 'mat'):
        np.mat = np.asmatrix
    fortran = types.ModuleType('fortran')
    fortran.EMUstack = types.ModuleType('EMUstack')
    sys.modules['fortran'] = fortran
    sys.modules['fortran.EMUstack'] = fortran.EMUstack
    mpl = types.ModuleType('matplotlib')
    mpl.use = lambda *a, **k: None
    plt = types.ModuleType('matplotlib.pyplot')
    mpl.pyplot = plt
    sys.modules['matplotlib'] = mpl
    sys.modules['matplotlib.pyplot'] = plt
    for sub in ('matplotlib.cm', 'matplotlib.colors', 'matplotlib.mlab',
                'matplotlib.gridspec', 'matplotlib.ticker', 'mpl_toolkits',
                'mpl_toolkits.axes_grid1'):
        sys.modules[sub] = types.ModuleType(sub)
    os.chdir(os.path.join(REF, 'tests'))   # reference paths are relative
    sys.path.insert(0, os.path.join(REF, 'backend'))
    import objects
    import materials
    import stack
    import mode_calcs
    return objects, materials, stack, mode_calcs


def _arr(x):
    return np.asarray(x)


def save_case(name, d):
    path = os.path.join(HERE, name + '.npz')
    np.savez_compressed(path, **d)
    print('wrote', path, sum(v.nbytes for v in d.values()), 'bytes')


def record_stack(d, key, st, light, pol, incoming=None, shears=None):
    """Store the inputs and outputs of one reference Stack."""
    from mode_calcs import Anallo
    d[key + 'wl_nm'] = _arr(light.wl_nm)
    d[key + 'k_pll'] = _arr(light.k_pll)
    d[key + 'max_order'] = _arr(light.max_order_PWs)
    d[key + 'period'] = _arr(st.period)
    d[key + 'period_y'] = _arr(st.period_y)
    d[key + 'pol'] = np.array(pol)
    d[key + 'n_layers'] = _arr(len(st.layers))
    d[key + 'heights_nm'] = _arr(st.heights_nm())
    d[key + 'world_1d'] = _arr(bool(st.layers[0].structure.world_1d))
    if incoming is not None:
        d[key + 'incoming'] = _arr(incoming).reshape(-1)
    if shears is not None:
        d[key + 'shears'] = np.array([np.asarray(s, dtype=float) for s in shears])
    for i, lay in enumerate(st.layers):
        lk = key + 'lay%d_' % i
        if isinstance(lay, Anallo):
            d[lk + 'kind'] = np.array('film')
            d[lk + 'n'] = _arr(complex(lay.structure.material.n(light.wl_nm)))
            d[lk + 'loss'] = _arr(bool(lay.structure.loss))
            d[lk + 'num_prop'] = _arr(lay.num_prop_pw_per_pol)
            d[lk + 'specular_order'] = _arr(lay.specular_order)
        else:
            d[lk + 'kind'] = np.array('struct')
            if getattr(lay, '_golden_J', None) is not None:
                d[lk + 'J'] = _arr(lay.J)
                d[lk + 'J_dag'] = _arr(lay.J_dag)
        d[lk + 'k_z'] = _arr(lay.k_z)
        d[lk + 'R12'] = _arr(lay.R12)
        d[lk + 'T12'] = _arr(lay.T12)
        d[lk + 'R21'] = _arr(lay.R21)
        d[lk + 'T21'] = _arr(lay.T21)
    d[key + 'R_net'] = _arr(st.R_net)
    d[key + 'T_net'] = _arr(st.T_net)
    d[key + 'a_list'] = np.array([float(np.real(np.asarray(a)).ravel()[0]) for a in st.a_list])
    d[key + 't_list'] = np.array([float(np.real(np.asarray(a)).ravel()[0]) for a in st.t_list])
    d[key + 'r_list'] = np.array([float(np.real(np.asarray(a)).ravel()[0]) for a in st.r_list])
    for nm in ('vec_coef_down', 'vec_coef_up'):
        vs = [_arr(v).ravel() for v in getattr(st, nm)]
        d[key + nm] = np.concatenate(vs)
        d[key + nm + '_len'] = np.array([len(v) for v in vs])


def main():
    objects, materials, stack, mode_calcs = import_reference()
    Stack = stack.Stack
    Simmo = mode_calcs.Simmo

    def stub_simmo(structure, light, k_z, J=None, J_dag=None, rt=None):
        sim = Simmo(structure, light)
        sim.k_z = np.asarray(k_z)
        if J is not None:
            sim.J = np.asmatrix(J)
            sim.J_dag = np.asmatrix(J_dag)
            sim._golden_J = True
        else:
            sim._golden_J = None
        if rt is not None:
            air = sim.air_ref()
            mode_calcs._interfaces_i_have_known[id(air), id(sim)] = tuple(np.asmatrix(m) for m in rt)
        return sim

    # ---------------- case 0: 7-layer thin-film stack, recomputed ----------
    # tests/test_case_0_thin_film_multistack.py:46-103
    d = {}
    period = 1
    sup = objects.ThinFilm(period=period, height_nm='semi_inf',
                           material=materials.Material(3.5 + 0.0j), loss=False)
    f1 = objects.ThinFilm(period=period, height_nm=50,
                          material=materials.Material(3.6 + 0.27j), loss=True)
    f2 = objects.ThinFilm(period=period, height_nm=200, material=materials.Si_c, loss=True)
    mirror = objects.ThinFilm(period=period, height_nm=100, material=materials.Ag, loss=True)
    sub = objects.ThinFilm(period=period, height_nm='semi_inf',
                           material=materials.Air, loss=False)
    wls = np.linspace(400, 1000, 3)
    ref0 = np.load('ref/case_0.npz', allow_pickle=True, encoding='latin1')['stack_list']
    for p, wl in enumerate(wls):
        light = objects.Light(wl, max_order_PWs=1, theta=0.0, phi=0.0)
        lays = [sub.calc_modes(light), mirror.calc_modes(light), f1.calc_modes(light),
                f2.calc_modes(light), f1.calc_modes(light), f2.calc_modes(light),
                sup.calc_modes(light)]
        st = Stack(lays)
        st.calc_scat(pol='TM')
        record_stack(d, 'p%d_' % p, st, light, 'TM')
        d['p%d_stored_R_net' % p] = _arr(ref0[p]['R_net'])
        d['p%d_stored_T_net' % p] = _arr(ref0[p]['T_net'])
        for i, rl in enumerate(ref0[p]['layers']):
            for m in ('R12', 'T12', 'R21', 'T21', 'k_z'):
                d['p%d_stored_lay%d_%s' % (p, i, m)] = _arr(rl[m])
    d['n_points'] = _arr(len(wls))
    save_case('case_0', d)

    # ---------------- cases 1-5: replay stored nanostructure interfaces -----
    specs = {
        # case: (wavelengths, max_order, theta, phi, period, pol, sub, sup, heights, world_1d)
        1: ([500, 1000], 2, 0.0, 0.0, 600, 'TE', materials.SiO2, materials.Air, [2330], False),
        2: ([500.0], 1, 20, 40, 600, 'TE', materials.SiO2, materials.Air, [2330], False),
        3: ([700], 2, 0.0, 0.0, 500, 'TE', materials.SiO2, materials.Air, [2330], False),
        4: ([800.0], 6, 0.0, 0.0, 760, 'TE', materials.Air, materials.Air, [150, 900], True),
        5: ([1.11 * 940], 4, 5.0, 0.0, 940, 'TM', materials.Air, materials.Air, [200], False),
    }
    for case, (wls, mo, th, ph, per, pol, msub, msup, hs, w1d) in specs.items():
        d = {}
        stored = np.load('ref/case_%d.npz' % case, allow_pickle=True, encoding='latin1')['stack_list']
        for p, wl in enumerate(wls):
            light = objects.Light(wl, max_order_PWs=mo, theta=th, phi=ph)
            tf_sub = objects.ThinFilm(per, height_nm='semi_inf', world_1d=w1d,
                                      material=msub, loss=False)
            tf_sup = objects.ThinFilm(per, height_nm='semi_inf', world_1d=w1d,
                                      material=msup, loss=False)
            lays = [tf_sub.calc_modes(light)]
            rls = stored[p]['layers']
            for j, h in enumerate(hs):
                ns = objects.NanoStruct('1D_array' if w1d else '2D_array', per, 100,
                                        height_nm=h, make_mesh_now=False,
                                        mesh_file='none.mail', world_1d=w1d)
                rl = rls[1 + j]
                lays.append(stub_simmo(ns, light, rl['k_z'],
                                       rt=(rl['R12'], rl['T12'], rl['R21'], rl['T21'])))
            lays.append(tf_sup.calc_modes(light))
            st = Stack(lays)
            st.calc_scat(pol=pol)
            record_stack(d, 'p%d_' % p, st, light, pol)
            d['p%d_stored_R_net' % p] = _arr(stored[p]['R_net'])
            d['p%d_stored_T_net' % p] = _arr(stored[p]['T_net'])
        d['n_points'] = _arr(len(wls))
        # txt goldens of the reference (tests/ref/case_N/*.txt), second column
        txtdir = 'ref/case_%d' % case
        if os.path.isdir(txtdir):
            for fn in sorted(os.listdir(txtdir)):
                if fn.endswith('.txt') and not fn.startswith('Efficiency'):
                    d['txt_' + fn[:-4]] = np.atleast_2d(np.loadtxt(os.path.join(txtdir, fn)))
        save_case('case_%d' % case, d)
    # txt goldens of case 0
    d = dict(np.load(os.path.join(HERE, 'case_0.npz')))
    for fn in sorted(os.listdir('ref/case_0')):
        if fn.endswith('.txt') and not fn.startswith('Efficiency'):
            d['txt_' + fn[:-4]] = np.atleast_2d(np.loadtxt(os.path.join('ref/case_0', fn)))
    save_case('case_0', d)

    # ---------------- synthetic nanostructured stacks ----------------------
    rng = np.random.default_rng(20261203)

    def synth_struct(light, per, M, P, h, scale=0.3):
        ns = objects.NanoStruct('2D_array', per, 240, height_nm=h, make_mesh_now=False,
                                mesh_file='none.mail')
        k0 = 2 * np.pi / (light.wl_nm / per)
        kz = rng.uniform(0, 2 * k0, M) + 1j * rng.uniform(0, 0.1 * k0, M)
        J = scale * (rng.standard_normal((P, M)) + 1j * rng.standard_normal((P, M)))
        Jd = scale * (rng.standard_normal((M, P)) + 1j * rng.standard_normal((M, P)))
        return stub_simmo(ns, light, kz, J=J, J_dag=Jd)

    # (a) config-1 shape: substrate 1.46 / one array (P=58, M=60) / air, TE
    d = {}
    per = 600
    sub = objects.ThinFilm(per, height_nm='semi_inf', material=materials.Material(1.46 + 0j), loss=False)
    sup = objects.ThinFilm(per, height_nm='semi_inf', material=materials.Air, loss=False)
    wls = [400.0, 650.0, 900.0]
    for p, wl in enumerate(wls):
        light = objects.Light(wl, max_order_PWs=3, theta=0.0, phi=0.0)
        lays = [sub.calc_modes(light), synth_struct(light, per, 60, 58, 100.0), sup.calc_modes(light)]
        st = Stack(lays)
        st.calc_scat(pol='TE')
        record_stack(d, 'p%d_' % p, st, light, 'TE')
    d['n_points'] = _arr(len(wls))
    save_case('synth_config1', d)

    # (b) M < P interface, two arrays with a spacer film, shears, pol 'un'
    d = {}
    per = 700
    sub = objects.ThinFilm(per, height_nm='semi_inf', material=materials.Material(1.46 + 0j), loss=False)
    spacer = objects.ThinFilm(per, height_nm=35.0, material=materials.Material(2.1 + 0.01j), loss=True)
    sup = objects.ThinFilm(per, height_nm='semi_inf', material=materials.Air, loss=False)
    light = objects.Light(720.0, max_order_PWs=2, theta=12.0, phi=30.0)
    P = 2 * len(sub.calc_modes(light).k_z) // 2
    lays = [sub.calc_modes(light), synth_struct(light, per, 20, P, 80.0),
            spacer.calc_modes(light), synth_struct(light, per, 30, P, 120.0),
            sup.calc_modes(light)]
    shears = ([0.0, 0.0], [0.1, 0.2], [0.15, 0.05], [0.3, 0.4], [0.0, 0.1])
    st = Stack(lays, shears=shears)
    st.calc_scat(pol='un')
    record_stack(d, 'p0_', st, light, 'un', shears=shears)
    d['n_points'] = _arr(1)
    save_case('synth_shear', d)

    # (c) 10-film stacks of the batched thin-film workload (period 500,
    #     max order 5), a few spectral points, several polarisations
    d = {}
    per = 500
    L = 10
    hs = rng.uniform(20, 300, L)
    nr = rng.uniform(1.3, 4.0, L)
    ki = rng.uniform(0, 0.5, L)
    films = [objects.ThinFilm(per, height_nm=float(hs[i]),
                              material=materials.Material(complex(nr[i], ki[i])), loss=True)
             for i in range(L)]
    sub = objects.ThinFilm(per, height_nm='semi_inf', material=materials.Material(1.46 + 0j), loss=False)
    sup = objects.ThinFilm(per, height_nm='semi_inf', material=materials.Air, loss=False)
    pols = ['TE', 'TM', 'un', 'R Circ', 'L Circ', 'TE']
    npts = len(pols)
    wls_c = rng.uniform(350, 1100, npts)
    th_c = rng.uniform(0, 60, npts)
    ph_c = rng.uniform(0, 90, npts)
    for p in range(npts):
        light = objects.Light(float(wls_c[p]), max_order_PWs=5, theta=float(th_c[p]), phi=float(ph_c[p]))
        lays = [sub.calc_modes(light)] + [f.calc_modes(light) for f in films] + [sup.calc_modes(light)]
        st = Stack(lays)
        st.calc_scat(pol=pols[p])
        record_stack(d, 'p%d_' % p, st, light, pols[p])
        d['p%d_theta' % p] = _arr(th_c[p])
        d['p%d_phi' % p] = _arr(ph_c[p])
    d['n_points'] = _arr(npts)
    save_case('films10', d)

    # (d) edge cases: custom incoming amplitudes; lossy substrate (no
    #     propagating orders); a stack with a single finite layer; normal
    #     incidence given by k_parallel (Wood anomaly branch)
    d = {}
    per = 450
    p = 0
    light = objects.Light(610.0, max_order_PWs=2, theta=33.0, phi=61.0)
    sub = objects.ThinFilm(per, height_nm='semi_inf', material=materials.Material(1.5 + 0j), loss=False)
    mid = objects.ThinFilm(per, height_nm=140.0, material=materials.Material(2.6 + 0.2j), loss=True)
    mid2 = objects.ThinFilm(per, height_nm=60.0, material=materials.Material(1.9 + 0.0j), loss=False)
    sup = objects.ThinFilm(per, height_nm='semi_inf', material=materials.Material(1.2 + 0j), loss=False)
    lays = [sub.calc_modes(light), mid.calc_modes(light), mid2.calc_modes(light), sup.calc_modes(light)]
    Pn = len(lays[0].k_z)
    inc = rng.standard_normal(Pn) + 1j * rng.standard_normal(Pn)
    st = Stack(lays)
    st.calc_scat(pol='TE', incoming_amplitudes=np.asmatrix(inc).T)
    record_stack(d, 'p%d_' % p, st, light, 'TE', incoming=inc)
    p += 1
    # lossy substrate: no propagating orders in the substrate
    lossy_sub = objects.ThinFilm(per, height_nm='semi_inf', material=materials.Material(1.5 + 0.3j), loss=True)
    light = objects.Light(500.0, max_order_PWs=1, theta=10.0, phi=20.0)
    lays = [lossy_sub.calc_modes(light), mid.calc_modes(light), sup.calc_modes(light)]
    st = Stack(lays)
    st.calc_scat(pol='TM')
    record_stack(d, 'p%d_' % p, st, light, 'TM')
    p += 1
    # Wood anomaly: period 1, k_parallel = (0.25, 0), air, and a wavelength
    # for which k^2 - alpha^2 - beta^2 is exactly 0.0 for order (1, 0)
    alpha = 0.25 + 2 * np.pi
    wl_w = 2 * np.pi / alpha
    while (np.complex128(2 * np.pi / wl_w) ** 2 - alpha ** 2 - 0.0 ** 2) != 0:
        wl_w = np.nextafter(wl_w, 2.0)
    light = objects.Light(float(wl_w), max_order_PWs=1, k_parallel=[0.25, 0.0])
    sub = objects.ThinFilm(1, height_nm='semi_inf', material=materials.Material(1.5 + 0j), loss=False)
    film = objects.ThinFilm(1, height_nm=0.4, material=materials.Material(2.5 + 0.1j), loss=True)
    sup = objects.ThinFilm(1, height_nm='semi_inf', material=materials.Air, loss=False)
    lays = [sub.calc_modes(light), film.calc_modes(light), sup.calc_modes(light)]
    st = Stack(lays)
    st.calc_scat(pol='TE')
    record_stack(d, 'p%d_' % p, st, light, 'TE')
    d['p%d_air_kz' % p] = _arr(light._air_ref(1.0, 1.0, False).k_z)
    p += 1
    d['n_points'] = _arr(p)
    save_case('edge_cases', d)

    # (e) dense interface alone at several shapes (M > P, M < P)
    d = {}
    per = 600
    shapes = [(58, 60), (58, 40), (26, 46)]
    for q, (P_, M_) in enumerate(shapes):
        mo = 3 if P_ == 58 else 2
        light = objects.Light(700.0 + 30 * q, max_order_PWs=mo, theta=7.0, phi=11.0)
        air = light._air_ref(float(per), float(per), False)
        sim = synth_struct(light, per, M_, len(air.k_z), 50.0)
        R12, T12, R21, T21 = mode_calcs.r_t_mat_tf_ns(air, sim)
        d['q%d_Z_air' % q] = _arr(air.Z())
        d['q%d_air_kz' % q] = _arr(air.k_z[:len(air.k_z) // 2])
        d['q%d_wl_norm' % q] = _arr(air.wl_norm())
        d['q%d_J' % q] = _arr(sim.J)
        d['q%d_J_dag' % q] = _arr(sim.J_dag)
        for nm, m in (('R12', R12), ('T12', T12), ('R21', R21), ('T21', T21)):
            d['q%d_%s' % (q, nm)] = _arr(m)
    d['n_shapes'] = _arr(len(shapes))
    save_case('interfaces', d)


if __name__ == '__main__':
    main()
