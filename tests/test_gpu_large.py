"""GPU parity of the dense GSM path at the large sizes of the nanostructured
workloads, against the CPU oracle (a numpy restatement of the reference's
FP64 algorithm: backend/mode_calcs.py:480-515 for the interfaces,
backend/stack.py:196-426 for the cascade and the fluxes).

* Four cylinder-array layers at period 700 nm, max order 10 (Npw = 309,
  P = 618) with M = 400 Bloch modes each, through the drop-in
  ``Stack.calc_scat`` under the automatic dense rule: D = max(P, M) >= 256
  takes the multi-CTA cascade and the multi-CTA interfaces with the LU panel
  on a thread-block cluster.
* One uneven batch (``emu_stack_var_batch``, one persistent launch) that
  holds a P = 882 stack with two M = 902 arrays beside smaller stacks.

Layers get seeded synthetic Bloch modes (complex normal J, J_dag of scale
0.25 / sqrt(P), k_z with Re U(0, 2 k0), Im U(0, 0.1 k0)).  With these inputs a
relative perturbation of the J entries is amplified 2e3- to 6e3-fold into
R_net and T_net (measured on the oracle), and the rounding of LU
factorisations of order 600 amounts to a relative perturbation of about
1e-13, so FP64 results computed in different orders differ by up to about
1e-10 of the largest entry.  The tests hold every entry to rtol 1e-9 with an
absolute floor of 1e-9 x max(1, max |entry|) (a normwise relative bar of
1e-9; the product bar is 1e-6 absolute).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _close(got, ref, msg):
    got, ref = np.asarray(got), np.asarray(ref)
    atol = 1e-9 * max(1.0, float(np.abs(ref).max()) if ref.size else 1.0)
    np.testing.assert_allclose(got, ref, rtol=1e-9, atol=atol, err_msg=msg)


def _synth_modes(rng, P, M, k0):
    s = 0.25 / np.sqrt(P)
    kz = rng.uniform(0, 2 * k0, M) + 1j * rng.uniform(0, 0.1 * k0, M)
    J = s * (rng.standard_normal((P, M)) + 1j * rng.standard_normal((P, M)))
    Jd = s * (rng.standard_normal((M, P)) + 1j * rng.standard_normal((M, P)))
    return kz, J, Jd


def _build(seed, wl, period, max_order, Ms, theta=0.0, phi=0.0):
    """The same stack as drop-in objects and as oracle layers: substrate
    n = 1.46, arrays (M > 0) or films (M = 0) bottom to top, air on top."""
    from oracle import gsm_oracle as O
    from emustack_b200 import materials, objects
    rng = np.random.default_rng(seed)
    light = objects.Light(wl, max_order_PWs=max_order, theta=theta, phi=phi)
    kp = light.k_pll
    air = O.make_air_ref(wl, kp, period, period, max_order, False)
    P = len(air.k_z)
    k0 = 2 * np.pi / (wl / period)
    sub = objects.ThinFilm(period, height_nm='semi_inf', material=materials.Material(1.46 + 0j), loss=False)
    sup = objects.ThinFilm(period, height_nm='semi_inf', material=materials.Air, loss=False)
    lays = [sub.calc_modes(light)]
    olays = [O.film_layer(1.46 + 0j, wl, kp, period, air, None, period, max_order, False, False)]
    hs = []
    for M in Ms:
        h = float(rng.uniform(50, 200))
        hs.append(h)
        if M:
            kz, J, Jd = _synth_modes(rng, P, M, k0)
            ns = objects.NanoStruct('2D_array', period, float(rng.uniform(100, 400)), height_nm=h)
            lays.append(ns.calc_modes(light, k_z=kz, J=J, J_dag=Jd))
            olays.append(O.OracleLayer('struct', kz, h, J=J, J_dag=Jd))
        else:
            n = complex(rng.uniform(1.3, 4.0), rng.uniform(0, 0.5))
            f = objects.ThinFilm(period, height_nm=h, material=materials.Material(n))
            lays.append(f.calc_modes(light))
            olays.append(O.film_layer(n, wl, kp, period, air, h, period, max_order, False, True))
    lays.append(sup.calc_modes(light))
    olays.append(O.film_layer(1.0 + 0j, wl, kp, period, air, None, period, max_order, False, False))
    return lays, olays, air, hs, P


@pytest.mark.parametrize('wl', [600.0, 850.0])
def test_four_arrays_P618_M400_match_oracle(wl):
    """Config-3 shape through Stack.calc_scat (multi-CTA dense path)."""
    from oracle import gsm_oracle as O
    from emustack_b200.stack import Stack
    lays, olays, air, hs, P = _build(int(wl), wl, 700.0, 10, [400] * 4)
    assert P == 618
    st = Stack(lays)
    st.calc_scat(pol='TE')
    ref = O.calc_scat(olays, air, 700.0, pol='TE', heights_nm=hs)
    _close(st.R_net, ref.R_net, 'R_net')
    _close(st.T_net, ref.T_net, 'T_net')
    for k in ('a_list', 't_list', 'r_list'):
        _close(np.asarray(getattr(st, k), float), np.asarray(getattr(ref, k), float), k)
    for i, (R12, T12, R21, T21) in enumerate(ref.interfaces):
        for nm, m in (('R12', R12), ('T12', T12), ('R21', R21), ('T21', T21)):
            _close(getattr(st.layers[i], nm), m, 'layer %d %s' % (i, nm))
    for a, b in zip(st.vec_coef_down, ref.vec_coef_down):
        _close(np.ravel(a), np.ravel(b), 'vec_coef_down')


def test_uneven_batch_with_P882_stack_matches_oracle():
    """One emu_stack_var_batch launch: a P = 882 stack (two M = 902 arrays
    and a film) beside smaller stacks of other shapes; each stack against
    the oracle."""
    from oracle import gsm_oracle as O
    from emustack_b200.dense import StackVarSolver, VarStack, layer_interface
    specs = [(7, 640.0, 12, [902, 0, 902]), (8, 720.0, 3, [60, 0]), (9, 500.0, 5, [0, 182, 0, 182]),
             (10, 910.0, 7, [150])]
    stacks, refs, keep = [], [], []
    for seed, wl, mo, Ms in specs:
        lays, olays, air_o, hs, P = _build(seed, wl, 500.0, mo, Ms, theta=20.0, phi=30.0)
        air = lays[-1].air_ref()
        dev_lays = []
        for i, lay in enumerate(lays):
            R12, T12, R21, T21, dense = layer_interface(air, lay)
            kz = hn = None
            if 0 < i < len(lays) - 1:
                kz = torch.tensor(np.asarray(lay.k_z), dtype=torch.complex128, device='cuda')
                hn = hs[i - 1] / 500.0
            dev_lays.append((R12[0], T12[0], R21[0], T21[0], dense, kz, 0.0 if hn is None else hn))
        keep.append(lays)
        top, sub = lays[-1], lays[0]
        stacks.append(VarStack(dev_lays, P, pol='TM', spec=int(top.specular_order),
                               num_prop=[air.num_prop_pw_per_pol, top.num_prop_pw_per_pol,
                                         sub.num_prop_pw_per_pol]))
        refs.append(O.calc_scat(olays, air_o, 500.0, pol='TM', heights_nm=hs))
    assert max(s.P for s in stacks) == 882
    out = StackVarSolver().solve(stacks, want_fluxes=True)
    torch.cuda.synchronize()
    h = {k: v.cpu().numpy() for k, v in out.items() if torch.is_tensor(v)}
    for i, (s, ref) in enumerate(zip(stacks, refs)):
        P, L = s.P, len(s.layers)
        ro, lo = int(out['rnet_off'][i]), int(out['list_off'][i])
        assert int(h['info'][i]) == 0
        _close(h['R_net'][ro:ro + P * P].reshape(P, P), ref.R_net, 'stack %d R_net' % i)
        _close(h['T_net'][ro:ro + P * P].reshape(P, P), ref.T_net, 'stack %d T_net' % i)
        _close(h['a_list'][lo:lo + L - 1], np.asarray(ref.a_list, float), 'stack %d a_list' % i)
        _close(h['t_list'][lo:lo + L - 1], np.asarray(ref.t_list, float), 'stack %d t_list' % i)
        _close(h['r_list'][i], float(ref.r_list[0]), 'stack %d r_list' % i)


def test_tensor_core_J_at_config3_size():
    """The split-TF32 x3 tensor-core J / J_dag at full config-3 size (20 000
    P2 triangles, M = 400 Bloch modes, period 700 nm, max order 10:
    K = 12 nel = 240 000) against the FP64 path on the same complex64
    fields.  The tensor cores accumulate in FP32, which drifts toward zero
    by about 7e-9 x K relative; the kernel starts a fresh accumulation every
    256 K values and sums the chunk results in FP32 within a split (the
    splits in FP64), so the J entries stay within 1e-5 of max |J| (measured
    1.8e-6)."""
    from emustack_b200 import objects
    from emustack_b200.films import grating_orders
    from emustack_b200.mesh import square_cell
    from emustack_b200.overlap import DeviceMesh, overlap_batch
    period, mo, M, wl = 700.0, 10, 400, 650.0
    mesh = square_cell(100, radius=0.3)
    assert mesh.nel == 20000
    dev = torch.device('cuda')
    g = torch.Generator(device='cuda').manual_seed(3)
    shape = (1, mesh.nel, M, 13, 3)
    cr = lambda: torch.complex(torch.randn(shape, dtype=torch.float32, device=dev, generator=g),
                               torch.randn(shape, dtype=torch.float32, device=dev, generator=g))
    s1_32, s2_32 = cr(), cr()
    px, py = grating_orders(mo, period, period)
    light = objects.Light(wl, max_order_PWs=mo, theta=0.0, phi=0.0)
    bloch = torch.tensor(np.asarray(light.k_pll * period).reshape(1, 2), device=dev)
    k0 = torch.tensor([2 * np.pi / (wl / period)], dtype=torch.float64, device=dev)
    dm = DeviceMesh(mesh)
    Jt, Jdt, _ = overlap_batch(dm, px, py, mo, bloch, k0, s1_32, s2_32, precision='tf32x3')
    Jt, Jdt = Jt[0].cpu().numpy(), Jdt[0].cpu().numpy()
    s1, s2 = s1_32.to(torch.complex128), s2_32.to(torch.complex128)
    del s1_32, s2_32
    J6, Jd6, _ = overlap_batch(dm, px, py, mo, bloch, k0, s1, s2, precision='fp64')
    J6, Jd6 = J6[0].cpu().numpy(), Jd6[0].cpu().numpy()
    del s1, s2
    torch.cuda.empty_cache()
    for a, b in ((Jt, J6), (Jdt, Jd6)):
        assert np.abs(a - b).max() <= 1e-5 * np.abs(b).max()
