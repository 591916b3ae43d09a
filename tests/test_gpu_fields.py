"""GPU parity of the field reconstruction (emu_pw_fields,
emu_bloch_fields_plane) and of the reference-facing field / spectra writers.

* With the reference's own layer data and amplitudes (tests/golden/
  fields.npz, made by the reference's field_values,
  backend/plotting.py:2857-2996), the kernel returns the reference's fields
  to 1e-13 of their largest magnitude.
* Through this package end to end (objects, Stack.calc_scat on the GPU,
  fields.field_values), the fields agree with the reference's to 1e-9 and
  the spectra files with the reference's files to their printed digits.
* Batched over points of a FilmStackSolver solve, the fields match the
  oracle, and the tangential field is continuous across every interface of
  12-layer stacks with 81 orders per polarisation.
* Bloch-mode node fields match the oracle restatement of field_value_plane
  (backend/fortran/field_value_plane.f:6-132) to 1e-13.
"""
import os

import numpy as np
import pytest
import torch

from oracle import fields_oracle as F

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, 'golden', 'fields.npz'))
KEYS = [str(k) for k in GOLD['names']]


def _ref_layer(key, i):
    d = GOLD
    L = len(d[key + 'n'])
    lk = key + 'lay%d_' % i
    row = L - 1 - i
    h = None if i in (0, L - 1) else d[key + 'heights_nm'][i - 1] / float(d[key + 'period'])
    return dict(alphas=d[lk + 'alphas'], betas=d[lk + 'betas'], sort_order=d[lk + 'sort_order'],
                kz=d[lk + 'kz'], n=complex(d[lk + 'n']), vec_coef_down=d[key + 'vec_coef_down'][row],
                vec_coef_up=None if i == 0 else d[key + 'vec_coef_up'][row],
                height_norm=h, substrate=(i == 0))


@pytest.mark.parametrize('key', KEYS)
def test_kernel_reproduces_reference_fields_from_reference_amplitudes(key):
    from emustack_b200.fields import pw_fields
    for i in range(len(GOLD[key + 'n'])):
        lk = key + 'lay%d_' % i
        xyz = GOLD[lk + 'xyz'].copy()
        if bool(GOLD[key + 'world_1d']):
            xyz[:, 1] = 0.0                      # field_values zeroes y in 1D worlds
        E, Eabs = pw_fields(x=xyz[:, 0], y=xyz[:, 1], z=xyz[:, 2], **_ref_layer(key, i))
        ref = GOLD[lk + 'E']
        scale = np.abs(ref).max()
        np.testing.assert_allclose(E[0].cpu().numpy(), ref, rtol=0, atol=1e-13 * scale, err_msg=lk)
        np.testing.assert_allclose(Eabs[0].cpu().numpy(), GOLD[lk + 'E_tot'].real, rtol=0, atol=1e-13 * scale)


def _our_stacks(name):
    from emustack_b200 import materials, objects
    from emustack_b200.stack import Stack
    out = []
    for key in [k for k in KEYS if k.startswith(name + '_')]:
        d = GOLD
        per, w1d = float(d[key + 'period']), bool(d[key + 'world_1d'])
        th, ph = d[key + 'theta_phi']
        light = objects.Light(float(d[key + 'wl_nm']), max_order_PWs=int(d[key + 'max_order']),
                              theta=float(th), phi=float(ph))
        np.testing.assert_allclose(np.asarray(light.k_pll, float), d[key + 'k_pll'], rtol=1e-15)
        ns, loss, hs = d[key + 'n'], d[key + 'loss'], d[key + 'heights_nm']
        L = len(ns)
        films = [objects.ThinFilm(period=per, height_nm=('semi_inf' if i in (0, L - 1) else float(hs[i - 1])),
                                  world_1d=w1d, material=materials.Material(complex(ns[i])), loss=bool(loss[i]))
                 for i in range(L)]
        st = Stack([f.calc_modes(light) for f in films])
        st.calc_scat(pol=str(d[key + 'pol']))
        out.append((key, st))
    return out


@pytest.mark.parametrize('name', ['s2d', 's2c', 's1d'])
def test_field_values_end_to_end_match_the_reference(name, tmp_path, monkeypatch):
    from emustack_b200.fields import field_values, t_r_a_write_files
    monkeypatch.chdir(tmp_path)
    stacks = _our_stacks(name)
    for key, st in stacks:
        for i in range(len(st.layers)):
            lk = key + 'lay%d_' % i
            sp = field_values([st], lay_interest=i, xyz_values=[tuple(q) for q in GOLD[lk + 'xyz']])
            Ex, Ey, Ez, Et = sp[0]
            ref = GOLD[lk + 'E']
            scale = np.abs(ref).max()
            np.testing.assert_allclose(np.array([Ex, Ey, Ez]), ref, rtol=0, atol=1e-9 * scale, err_msg=lk)
            np.testing.assert_allclose(Et, GOLD[lk + 'E_tot'], rtol=0, atol=1e-9 * scale)
    files = os.listdir('field_values')
    assert len([f for f in files if f.endswith('.npz')]) == sum(len(st.layers) for _, st in stacks)
    # the spectra files: the reference's names, numbers equal to the printed digits
    t_r_a_write_files([st for _, st in stacks], np.array([float(GOLD[k + 'wl_nm']) for k, _ in stacks]),
                      stack_label=7)
    for fn, text in zip(GOLD[name + '_txt_names'], GOLD[name + '_txt_text']):
        got = np.loadtxt(str(fn))
        ref = np.loadtxt(str(text).splitlines())
        np.testing.assert_allclose(got, ref, rtol=0, atol=2e-11, err_msg=str(fn))


def test_fields_in_plane_grid_matches_the_oracle(tmp_path, monkeypatch):
    from emustack_b200.fields import fields_in_plane
    monkeypatch.chdir(tmp_path)
    (key, st), = _our_stacks('s2c')
    per = float(GOLD[key + 'period'])
    z_nm = [0.0, 25.0, 60.0]
    res = fields_in_plane([st], lay_interest=1, z_values=z_nm, nu_calc_pts=20)[0]
    assert res['E_x'].shape == (21, 21, 3)
    lay = st.layers[1]
    S = lay.structure.num_pw_per_pol
    G = F.pw_field_grid(lay.alphas, lay.betas, lay.sort_order, np.asarray(lay.k_z)[:S], complex(lay.n()),
                        np.asarray(st.vec_coef_down[1]).ravel(), np.asarray(st.vec_coef_up[1]).ravel(),
                        res['x'], res['y'], np.array(z_nm) / per, height_norm=60.0 / per)
    for c, k in enumerate(('E_x', 'E_y', 'E_z')):
        scale = np.abs(G[c]).max() + 1e-300
        np.testing.assert_allclose(res[k], G[c], rtol=0, atol=1e-13 * max(scale, np.abs(G[0]).max()))
    assert os.path.isdir('in_plane_fields') and os.listdir('in_plane_fields')
    with pytest.raises(ValueError):
        fields_in_plane([st], lay_interest=1, z_values=[61.0])


def _film_batch(B, L, max_order, seed, world_1d=False):
    from emustack_b200.films import FilmStackSolver
    rng = np.random.default_rng(seed)
    period = 500.0
    s = FilmStackSolver(L, max_order, period, world_1d=world_1d)
    dev = s.device
    wl = rng.uniform(400, 1000, B)
    th, ph = np.radians(rng.uniform(1, 50, B)), np.radians(rng.uniform(0, 90, B))
    k = 2 * np.pi / wl
    kp = np.stack([k * np.sin(th) * np.cos(ph), k * np.sin(th) * np.sin(ph)], 1)
    if world_1d:
        kp[:, 1] = 0.0
    n = np.concatenate([np.full((B, 1), 1.46), rng.uniform(1.3, 3.5, (B, L - 2)) + 1j * rng.uniform(0, 0.3, (B, L - 2)),
                        np.ones((B, 1))], 1)
    hs = rng.uniform(30, 250, L - 2)
    out = s.solve(torch.tensor(wl, device=dev), torch.tensor(kp, device=dev),
                  torch.tensor(n, dtype=torch.complex128, device=dev), torch.tensor(hs, device=dev), pol='un',
                  want=('kz', 'vec_coef', 'sort_order'))
    return s, out, kp, n, hs


@pytest.mark.parametrize('world_1d', [False, True])
def test_batched_fields_match_the_oracle(world_1d):
    from emustack_b200.fields import film_batch_fields
    from emustack_b200.films import grating_orders
    B, L, mo = 24, 5, 3
    s, out, kp, n, hs = _film_batch(B, L, mo, seed=11, world_1d=world_1d)
    px, py = grating_orders(mo, 500.0, 500.0, world_1d)
    rng = np.random.default_rng(2)
    for layer in range(L):
        zmax = 0.3 if layer in (0, L - 1) else hs[layer - 1] / 500.0
        pts = np.column_stack([rng.uniform(0, 1, 7), rng.uniform(0, 1, 7), rng.uniform(0, zmax, 7)])
        E, Eabs = film_batch_fields(s, out, kp, n, layer, pts[:, 0], pts[:, 1], pts[:, 2], heights_nm=hs)
        E = E.cpu().numpy()
        o = {k: v.cpu().numpy() for k, v in out.items()}
        row = L - 1 - layer
        for b in range(0, B, 5):
            alphas = kp[b, 0] * 500.0 + px * 2 * np.pi
            betas = kp[b, 1] * 500.0 + np.asarray(py) * 2 * np.pi     # py = 0 in a 1D world
            ref = F.pw_field_points(alphas, betas, o['sort_order'][b], o['kz'][b, layer], n[b, layer],
                                    o['vec_coef_down'][b, row],
                                    None if layer == 0 else o['vec_coef_up'][b, row], pts,
                                    height_norm=None if layer in (0, L - 1) else hs[layer - 1] / 500.0,
                                    substrate=(layer == 0), world_1d=False)
            scale = np.abs(np.array(ref[:3])).max()
            np.testing.assert_allclose(E[b], np.array(ref[:3]), rtol=0, atol=1e-12 * scale)


def test_tangential_field_continuous_at_config2_size():
    """12 layers, max order 5 (81 orders per polarisation): E_x, E_y at the
    top of every layer equal those at the bottom of the next, every point."""
    from emustack_b200.fields import film_batch_fields
    B, L = 64, 12
    s, out, kp, n, hs = _film_batch(B, L, 5, seed=12)
    rng = np.random.default_rng(3)
    x, y = rng.uniform(0, 1, 9), rng.uniform(0, 1, 9)
    for i in range(L - 1):
        ztop = 0.0 if i == 0 else hs[i - 1] / 500.0
        below, _ = film_batch_fields(s, out, kp, n, i, x, y, np.full(9, ztop), heights_nm=hs)
        above, _ = film_batch_fields(s, out, kp, n, i + 1, x, y, np.zeros(9), heights_nm=hs)
        below, above = below[:, :2].cpu().numpy(), above[:, :2].cpu().numpy()
        scale = np.abs(below).max(axis=(1, 2), keepdims=True)
        assert np.all(np.abs(below - above) <= 1e-9 * scale), 'interface %d' % i


@pytest.mark.parametrize('nel,M,B', [(300, 40, 2), (2048, 60, 1)])
def test_bloch_plane_matches_the_oracle(nel, M, B):
    from emustack_b200.fields import bloch_fields_plane
    rng = np.random.default_rng(nel)
    sol = rng.normal(size=(B, nel, M, 13, 3)) + 1j * rng.normal(size=(B, nel, M, 13, 3))
    kz = rng.uniform(0.5, 3, (B, M)) + 1j * rng.uniform(0, 0.5, (B, M))
    vc = rng.normal(size=(B, 2 * M)) + 1j * rng.normal(size=(B, 2 * M))
    h = 0.4
    for hz in (0.0, 0.13, h):
        got = bloch_fields_plane(sol, kz, vc, h, hz).cpu().numpy()
        for b in range(B):
            ref = F.bloch_field_plane(sol[b], kz[b], vc[b], h, hz)
            np.testing.assert_allclose(got[b], ref, rtol=0, atol=1e-13 * np.abs(ref).max())


def test_bloch_plane_refuses_a_plane_outside_the_layer():
    import ctypes as C
    from emustack_b200 import _lib
    from emustack_b200.fields import bloch_fields_plane
    sol = np.zeros((4, 3, 13, 3), complex)
    with pytest.raises(ValueError):
        bloch_fields_plane(sol, np.ones((1, 3)), np.ones((1, 6)), 0.5, 0.6)
    d = _lib.EmuBlochFieldsPlane()
    d.n_stacks, d.n_modes, d.n_elements, d.h, d.hz = 1, 3, 4, 0.5, -0.1
    assert _lib.lib().emu_bloch_fields_plane(C.byref(d), None) == 1   # EMU_E_ARG before any launch


@pytest.mark.parametrize('nz,substrate', [(1, False), (5, False), (9, True)])
def test_grid_tables_match_the_term_by_term_points(nz, substrate):
    """The grid path (per-axis exponential tables and a contraction over
    orders, z in passes of 4, orders in stages of 64) equals the term-by-term
    point evaluation of the same grid."""
    from emustack_b200.fields import pw_fields
    from emustack_b200.films import grating_orders
    rng = np.random.default_rng(nz)
    B, mo = 3, 6
    px, py = grating_orders(mo, 500.0, 500.0, False)
    S = len(px)
    assert S > 64
    k0 = 2 * np.pi / rng.uniform(0.8, 2.0, B)
    alphas = rng.uniform(-0.3, 0.3, (B, 1)) + 2 * np.pi * px[None]
    betas = rng.uniform(-0.3, 0.3, (B, 1)) + 2 * np.pi * py[None]
    n = rng.uniform(1.2, 3.0, B) + 1j * rng.uniform(0, 0.2, B)
    kz = np.sqrt(((n * k0)[:, None] ** 2 - alphas ** 2 - betas ** 2).astype(complex))
    sort = np.argsort(-kz.real + kz.imag, axis=1, kind='stable').astype(np.int32)
    kz = np.take_along_axis(kz, sort, 1)
    vcd = rng.normal(size=(B, 2 * S)) + 1j * rng.normal(size=(B, 2 * S))
    vcu = rng.normal(size=(B, 2 * S)) + 1j * rng.normal(size=(B, 2 * S))
    h = rng.uniform(0.1, 0.4, B)
    xs, ys = np.linspace(0, 1, 7), np.linspace(0, 1, 6)
    zs = np.linspace(0, 0.1, nz)
    args = dict(alphas=alphas, betas=betas, sort_order=sort, kz=kz, n=n, vec_coef_down=vcd,
                vec_coef_up=vcu, height_norm=None if substrate else h, substrate=substrate)
    G, Gabs = pw_fields(x=xs, y=ys, z=zs, grid=True, **args)
    pts = np.array([(x, y, z) for x in xs for y in ys for z in zs])
    P, Pabs = pw_fields(x=pts[:, 0], y=pts[:, 1], z=pts[:, 2], grid=False, **args)
    G, P = G.cpu().numpy(), P.cpu().numpy()
    for b in range(B):
        scale = np.abs(P[b]).max()
        np.testing.assert_allclose(G[b], P[b], rtol=0, atol=1e-13 * scale)
    np.testing.assert_allclose(Gabs.cpu().numpy(), Pabs.cpu().numpy(), rtol=1e-12, atol=1e-13 * np.abs(P).max())


@pytest.mark.parametrize('name,no_incoming', [('s2d', False), ('s2c', True), ('s1d', False)])
def test_fields_vertically_matches_the_oracle(name, no_incoming, tmp_path, monkeypatch):
    """x-z slices through every film layer on fields_vertically's grids (z
    negative inside the substrate, the superstrate with or without the
    incident field) against the restatement of its loop."""
    from emustack_b200.fields import fields_vertically
    monkeypatch.chdir(tmp_path)
    (key, st), = _our_stacks(name)[:1]
    res = fields_vertically([st], factor_pts_vert=11, nu_pts_hori=12, semi_inf_height=0.5,
                            no_incoming=no_incoming)[0]
    assert os.path.exists('fields_vertically/stack_0.npz')
    L = len(st.layers)
    hs = st.heights_norm()
    h_list = [-0.5, 0.0] + list(np.cumsum(hs)) + [0.0]
    h_list[-1] = h_list[-2] + 0.5
    x = res['x']
    assert len(x) == 13
    for lay in range(L):
        ly = st.layers[lay]
        S = ly.structure.num_pw_per_pol
        ind_h = 0.5 if lay in (0, L - 1) else hs[lay - 1]
        nz = max(11, int(np.round(11 * np.real(np.max(np.asarray(ly.n()) ** 2)) * ind_h / ly.wl_norm())))
        z_range = np.linspace(-0.5, 0.0, nz) if lay == 0 else np.linspace(0.0, ind_h, nz)
        row = L - 1 - lay
        vcd = np.asarray(st.vec_coef_down[row]).ravel()
        if lay == L - 1 and no_incoming:
            vcd = np.zeros_like(vcd)
        vcu = None if lay == 0 else np.asarray(st.vec_coef_up[row]).ravel()
        betas = np.atleast_1d(np.asarray(ly.betas, float))
        betas = np.full(S, betas[0]) if betas.size == 1 else betas
        ref = F.vertical_slice(ly.alphas, betas, ly.sort_order, np.asarray(ly.k_z)[:S], complex(ly.n()), vcd, vcu,
                               x, z_range, h_norm=None if lay in (0, L - 1) else hs[lay - 1])
        scale = max(np.abs(r).max() for r in ref)
        for c, k in enumerate(('E_x_%d', 'E_y_%d', 'E_z_%d')):
            got = res[k % lay]
            assert got.shape == (13, nz)
            np.testing.assert_allclose(got, ref[c], rtol=0, atol=1e-13 * scale, err_msg='%s layer %d' % (k, lay))
