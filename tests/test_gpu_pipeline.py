"""The batched per-wavelength GSM chain (emustack_b200.pipeline): one batch
of wavelengths through film modes, adjoint normalisation, J / J_dag,
interfaces and the cascade equals the drop-in Stack path wavelength by
wavelength (FP64, rtol 1e-9), and its CUDA-graph replay equals the eager
run bit for bit, also after new inputs are loaded."""
import numpy as np
import pytest
import torch

from emustack_b200.mesh import square_cell

pytestmark = pytest.mark.gpu

PERIOD, MO, M, H = 600.0, 2, 30, 120.0


def _inputs(rng, B, nel):
    wl = rng.uniform(450, 850, B)
    sol1 = 0.02 * (rng.standard_normal((B, nel, M, 13, 3)) + 1j * rng.standard_normal((B, nel, M, 13, 3)))
    sol2 = 0.02 * (rng.standard_normal((B, nel, M, 13, 3)) + 1j * rng.standard_normal((B, nel, M, 13, 3)))
    k0 = 2 * np.pi / (wl / PERIOD)
    beta = rng.uniform(0, 2, (B, M)) * k0[:, None] + 1j * rng.uniform(0, 0.1, (B, M)) * k0[:, None]
    return wl, sol1, sol2, beta


def _drop_in(mesh, wl, s1, s2, beta, light_args):
    from emustack_b200 import materials, objects
    from emustack_b200.stack import Stack
    light = objects.Light(wl, max_order_PWs=MO, **light_args)
    ns = objects.NanoStruct('2D_array', PERIOD, 240, height_nm=H)
    sim = ns.calc_modes(light, k_z=beta, fields=dict(sol1=s1, sol2=s2, mesh=mesh))
    sub = objects.ThinFilm(PERIOD, height_nm='semi_inf', material=materials.Material(1.46 + 0j), loss=False)
    sup = objects.ThinFilm(PERIOD, height_nm='semi_inf', material=materials.Air, loss=False)
    st = Stack([sub.calc_modes(light), sim, sup.calc_modes(light)])
    st.calc_scat(pol='TE')
    return st, light


def test_pipeline_matches_drop_in_stack_and_graph_replay():
    from emustack_b200.pipeline import NanoStackPipeline
    rng = np.random.default_rng(21)
    mesh = square_cell(8, radius=0.3, jitter=0.15)
    B = 3
    wl, s1, s2, beta = _inputs(rng, B, mesh.nel)
    largs = dict(theta=7.0, phi=20.0)
    refs = [_drop_in(mesh, wl[b], s1[b], s2[b], beta[b], largs) for b in range(B)]
    kp = np.stack([np.asarray(l.k_pll, float) for _, l in refs])
    pl = NanoStackPipeline(mesh, PERIOD, MO, M, B, H)
    dev = torch.device('cuda')
    to = lambda a: torch.tensor(a, device=dev)
    pl.load(wl, kp, to(s1), to(s2), to(beta))
    eager = {k: v.clone() for k, v in pl.forward().items()}
    torch.cuda.synchronize()
    for b, (st, _) in enumerate(refs):
        np.testing.assert_allclose(eager['R_net'][b].cpu().numpy(), np.asarray(st.R_net), rtol=1e-9, atol=1e-11)
        np.testing.assert_allclose(eager['T_net'][b].cpu().numpy(), np.asarray(st.T_net), rtol=1e-9, atol=1e-11)
        np.testing.assert_allclose(eager['a_list'][b].cpu().numpy(), np.asarray(st.a_list, float),
                                   rtol=1e-9, atol=1e-11)
    out = pl.capture()
    pl.replay()
    torch.cuda.synchronize()
    for k in ('R_net', 'T_net', 'a_list', 't_list', 'r_list'):
        assert torch.equal(out[k], eager[k]), k
    # new inputs through the same graph
    wl2, t1, t2, beta2 = _inputs(rng, B, mesh.nel)
    pl.load(wl2, kp, to(t1), to(t2), to(beta2))
    pl.replay()
    torch.cuda.synchronize()
    replayed = {k: out[k].clone() for k in ('R_net', 'a_list')}
    pl.load(wl2, kp, to(t1), to(t2), to(beta2))
    again = pl.forward()
    torch.cuda.synchronize()
    for k in replayed:
        assert torch.equal(replayed[k], again[k]), k
    assert not torch.equal(replayed['R_net'], eager['R_net'])
