"""Device evaluation of the layers' refractive indices (emu_material_n_batch)
against the oracle's restatement of backend/materials.py (Material.n: constant,
scipy interp1d over tabulated data, Drude) with Anallo.n's loss flag, and a
wavelength sweep of a film stack with tabulated materials solved from the
device indices against the oracle."""
import numpy as np
import pytest
import torch

from oracle import gsm_oracle as G

pytestmark = pytest.mark.gpu


def _tables(rng):
    wl = np.sort(rng.uniform(300, 1200, 40))
    wl[0], wl[-1] = 300.0, 1200.0
    complex_tab = np.stack([wl, 1.5 + rng.uniform(0, 2.5, 40), rng.uniform(0, 0.6, 40)], axis=1)
    real_tab = np.stack([np.append(wl[:-2:2], 1200.0), 1.3 + rng.uniform(0, 1, 20)], axis=1)
    return complex_tab, real_tab


def test_material_indices_match_the_oracle():
    from emustack_b200.materials import Material, n_batch
    rng = np.random.default_rng(3)
    ct, rt = _tables(rng)
    specs = [1.46 + 0j, ct, rt, np.array([1.36e16, 1.05e14, 9.5]), 3.5 + 0.2j, ct]
    losses = [True, True, True, True, False, False]
    mats = [Material(s) for s in specs]
    wl = np.concatenate([rng.uniform(300, 1200, 500), ct[:, 0], rt[:, 0], [300.0, 1200.0]])
    out = n_batch(mats, torch.tensor(wl, device='cuda'), losses).cpu().numpy()
    for l, (s, loss) in enumerate(zip(specs, losses)):
        ref = np.array([G.material_n(s, w, loss) for w in wl], complex)
        np.testing.assert_allclose(out[:, l], ref, rtol=2e-15, atol=1e-15, err_msg='layer %d' % l)


def test_out_of_range_wavelength_raises():
    from emustack_b200.materials import Material, n_batch
    ct, _ = _tables(np.random.default_rng(4))
    with pytest.raises(ValueError):
        n_batch([Material(ct)], torch.tensor([250.0, 500.0], dtype=torch.float64, device='cuda'))


def test_sweep_of_tabulated_films_matches_the_oracle():
    """Wavelength sweep of a stack of tabulated films: indices on the
    device feed the film kernel directly."""
    from emustack_b200.films import FilmStackSolver
    from emustack_b200.materials import Material, n_batch
    rng = np.random.default_rng(5)
    ct, rt = _tables(rng)
    specs = [1.46 + 0j, ct, rt, ct, 1.0 + 0j]
    losses = [False, True, True, True, False]
    mats = [Material(s) for s in specs]
    B = 64
    wl = np.linspace(350.0, 1100.0, B)
    kp = np.array([G.k_parallel_from_angles(w, 25.0, 40.0) for w in wl])
    h = np.array([120.0, 60.0, 240.0])
    dev = torch.device('cuda')
    d_wl = torch.tensor(wl, device=dev)
    n = n_batch(mats, d_wl, losses)
    out = FilmStackSolver(len(mats), 4, 500.0).solve(d_wl, torch.tensor(kp, device=dev), n,
                                                     torch.tensor(h, device=dev), pol='TM')
    for b in range(0, B, 9):
        ns = [G.material_n(s, wl[b], lo) for s, lo in zip(specs, losses)]
        r = G.film_stack_point(ns, h, wl[b], kp[b], 500.0, max_order=4, pol='TM')
        np.testing.assert_allclose(out['R_net'][b].cpu().numpy(), np.diag(r.R_net), rtol=1e-9, atol=1e-10)
        np.testing.assert_allclose(out['a_list'][b].cpu().numpy(), np.asarray(r.a_list, float),
                                   rtol=1e-9, atol=1e-10)


def test_material_kernel_matches_the_reference_values():
    """emu_material_n_batch against the reference's own Material.n outputs
    (tests/golden/materials.npz): tabulated and constant bit for bit; Drude
    bit for bit wherever numpy's w**2 (the C library's pow) equals w*w.  At
    the few wavelengths where pow rounds w^2 to the other neighbour the
    kernel keeps the exact square and agrees to the conditioning of
    eps_inf - wp^2/(...), checked at 1e-13."""
    import os
    from emustack_b200.materials import Material, n_batch
    gold = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'materials.npz'))
    names = ['const', 'complex_tab', 'real_tab', 'drude']
    specs = [gold['spec_' + k] for k in names]
    mats = [Material(s.item() if s.shape == () else s) for s in specs]
    wl = gold['wl']
    out = n_batch(mats, torch.tensor(wl, device='cuda'), [True] * 4).cpu().numpy()
    for l, k in enumerate(names):
        ref = gold['n_' + k]
        if k == 'drude':
            w = (2 * np.pi * 299792458.0) / (wl * 1e-9)
            same = np.array([np.float64(x) ** 2 == x * x for x in w])
            assert same.sum() >= len(w) - 4
            np.testing.assert_array_equal(out[same, l], ref[same], err_msg=k)
            np.testing.assert_allclose(out[~same, l], ref[~same], rtol=1e-13, atol=0, err_msg=k)
        else:
            np.testing.assert_array_equal(out[:, l], ref, err_msg=k)
