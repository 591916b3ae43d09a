"""Tensor-core (tcgen05, split-TF32 x3, FP32 accumulation) path of the
overlap integrals: the GEMM alone against an FP64 product, J / J_dag against
the FP64 path, and the resulting R / T / A against the FP64 chain within the
product bar (1e-6 absolute)."""
import numpy as np
import pytest
import torch

from emustack_b200.mesh import square_cell

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('m,n,k,splits', [(1, 1, 1, 1), (128, 128, 32, 1), (130, 77, 100, 2),
                                          (618, 800, 4096, 8), (58, 120, 3000, 3)])
def test_tc_gemm_matches_fp64(m, n, k, splits):
    from emustack_b200.overlap import tc_gemm
    rng = np.random.default_rng(m + n + k)
    A = rng.standard_normal((m, k))
    B = rng.standard_normal((n, k))
    C = tc_gemm(torch.tensor(A, device='cuda'), torch.tensor(B, device='cuda'), splits).cpu().numpy()
    ref = A @ B.T
    # split-TF32 products: ~2^-21 relative per term, FP32 accumulation
    tol = 2e-6 * np.sqrt(k) + 1e-6
    np.testing.assert_allclose(C, ref, rtol=0, atol=tol * np.abs(A).max() * np.abs(B).max())


def _fields(rng, nel, nval):
    return rng.standard_normal((nel, nval, 13, 3)) + 1j * rng.standard_normal((nel, nval, 13, 3))


def test_overlap_tensor_cores_match_fp64():
    from emustack_b200.films import grating_orders
    from emustack_b200.overlap import DeviceMesh, overlap_batch
    rng = np.random.default_rng(9)
    mesh = square_cell(12, radius=0.3, jitter=0.2)
    mo, nval = 3, 40
    px, py = grating_orders(mo, 600.0, 600.0)
    s1 = torch.tensor(_fields(rng, mesh.nel, nval)[None], device='cuda')
    s2 = torch.tensor(_fields(rng, mesh.nel, nval)[None], device='cuda')
    bloch = torch.tensor([[0.13, -0.29]], dtype=torch.float64, device='cuda')
    k0 = torch.tensor([2 * np.pi / 1.21], dtype=torch.float64, device='cuda')
    dm = DeviceMesh(mesh)
    J64, Jd64, _ = overlap_batch(dm, px, py, mo, bloch, k0, s1, s2, precision='fp64')
    Jtc, Jdtc, _ = overlap_batch(dm, px, py, mo, bloch, k0, s1, s2, precision='tf32x3', elements_per_chunk=100)
    # split-TF32 drops lo*lo (~2^-22 relative per product); with FP32
    # accumulation the measured error is ~2e-6 of max|J| on random fields
    for a, b in ((Jtc, J64), (Jdtc, Jd64)):
        a, b = a.cpu().numpy(), b.cpu().numpy()
        assert np.abs(a - b).max() <= 5e-6 * np.abs(b).max()


def test_tensor_core_stack_within_product_bar():
    """R, T, A of a nanostructured stack with J / J_dag from the tensor-core
    path agree with the FP64 chain to 1e-6 absolute."""
    from emustack_b200 import objects, materials
    from emustack_b200.dense import interface_dense
    from emustack_b200.films import grating_orders
    from emustack_b200.overlap import DeviceMesh, overlap_batch
    from emustack_b200.stack import Stack
    rng = np.random.default_rng(10)
    period = 600.0
    mesh = square_cell(10, radius=0.25)
    light = objects.Light(650.0, max_order_PWs=3, theta=5.0, phi=15.0)
    nval = 70
    s1 = 0.02 * _fields(rng, mesh.nel, nval)
    s2 = 0.02 * _fields(rng, mesh.nel, nval)
    k0 = 2 * np.pi / (650.0 / period)
    kz = rng.uniform(0, 2 * k0, nval) + 1j * rng.uniform(0, 0.1 * k0, nval)
    px, py = grating_orders(3, period, period)
    dm = DeviceMesh(mesh)
    bloch = torch.tensor(np.asarray(light.k_pll * period).reshape(1, 2), device='cuda')
    k0t = torch.tensor([k0], dtype=torch.float64, device='cuda')
    S1 = torch.tensor(s1[None], device='cuda')
    S2 = torch.tensor(s2[None], device='cuda')
    out = {}
    for prec in ('fp64', 'tf32x3'):
        J, Jd, _ = overlap_batch(dm, px, py, 3, bloch, k0t, S1, S2, precision=prec)
        ns = objects.NanoStruct('2D_array', period, 240, height_nm=80.0)
        sim = ns.calc_modes(light, k_z=kz, J=J[0].cpu().numpy(), J_dag=Jd[0].cpu().numpy())
        sub = objects.ThinFilm(period, height_nm='semi_inf', material=materials.Material(1.46 + 0j), loss=False)
        sup = objects.ThinFilm(period, height_nm='semi_inf', material=materials.Air, loss=False)
        st = Stack([sub.calc_modes(light), sim, sup.calc_modes(light)])
        st.calc_scat(pol='TE')
        out[prec] = (np.asarray(st.a_list, float), np.asarray(st.t_list, float), np.asarray(st.r_list, float))
    for a, b in zip(out['fp64'], out['tf32x3']):
        np.testing.assert_allclose(b, a, rtol=0, atol=1e-6)


def test_overlap_tensor_cores_batched_problems():
    """Several wavelengths in one call: the tensor-core path runs them as one
    group (one launch per step for all problems) and matches the FP64 path
    problem by problem, including the adjoint normalisation factors."""
    from emustack_b200.films import grating_orders
    from emustack_b200.overlap import DeviceMesh, overlap_batch
    rng = np.random.default_rng(31)
    mesh = square_cell(10, radius=0.3, jitter=0.2)
    mo, nval, B = 3, 24, 3
    px, py = grating_orders(mo, 600.0, 600.0)
    s1 = torch.tensor(np.stack([_fields(rng, mesh.nel, nval) for _ in range(B)]), device='cuda')
    s2 = torch.tensor(np.stack([_fields(rng, mesh.nel, nval) for _ in range(B)]), device='cuda')
    bloch = torch.tensor(rng.uniform(-0.4, 0.4, (B, 2)), device='cuda')
    k0 = torch.tensor(2 * np.pi / rng.uniform(0.8, 1.6, B), device='cuda')
    scale = torch.tensor(rng.standard_normal((B, nval)) + 1j * rng.standard_normal((B, nval)), device='cuda')
    dm = DeviceMesh(mesh)
    J64, Jd64, inv64 = overlap_batch(dm, px, py, mo, bloch, k0, s1, s2, scale2=scale, precision='fp64')
    Jtc, Jdtc, invtc = overlap_batch(dm, px, py, mo, bloch, k0, s1, s2, scale2=scale, precision='tf32x3',
                                     elements_per_chunk=70)
    assert torch.equal(inv64, invtc)
    for a, b in ((Jtc, J64), (Jdtc, Jd64)):
        a, b = a.cpu().numpy(), b.cpu().numpy()
        for i in range(B):
            assert np.abs(a[i] - b[i]).max() <= 5e-6 * np.abs(b[i]).max()


def test_overlap_tensor_cores_complex64_fields():
    """Fields held as complex64 (the tensor-core operands are FP32 anyway):
    the same J / J_dag bit for bit as complex128 fields holding the same
    values, and the FP64 path's results to the tensor-core tolerance."""
    from emustack_b200.films import grating_orders
    from emustack_b200.overlap import DeviceMesh, overlap_batch
    rng = np.random.default_rng(33)
    mesh = square_cell(10, radius=0.3, jitter=0.2)
    mo, nval, B = 3, 24, 2
    px, py = grating_orders(mo, 600.0, 600.0)
    s1 = torch.tensor(np.stack([_fields(rng, mesh.nel, nval) for _ in range(B)]), device='cuda')
    s2 = torch.tensor(np.stack([_fields(rng, mesh.nel, nval) for _ in range(B)]), device='cuda')
    s1_32, s2_32 = s1.to(torch.complex64), s2.to(torch.complex64)
    s1_r, s2_r = s1_32.to(torch.complex128), s2_32.to(torch.complex128)   # same values, complex128
    bloch = torch.tensor(rng.uniform(-0.4, 0.4, (B, 2)), device='cuda')
    k0 = torch.tensor(2 * np.pi / rng.uniform(0.8, 1.6, B), device='cuda')
    dm = DeviceMesh(mesh)
    kw = dict(precision='tf32x3', elements_per_chunk=70, tc_splits=2)
    J32, Jd32, _ = overlap_batch(dm, px, py, mo, bloch, k0, s1_32, s2_32, **kw)
    Jr, Jdr, _ = overlap_batch(dm, px, py, mo, bloch, k0, s1_r, s2_r, **kw)
    assert torch.equal(J32, Jr) and torch.equal(Jd32, Jdr)
    J64, Jd64, _ = overlap_batch(dm, px, py, mo, bloch, k0, s1_r, s2_r, precision='fp64')
    for a, b in ((J32, J64), (Jd32, Jd64)):
        a, b = a.cpu().numpy(), b.cpu().numpy()
        assert np.abs(a - b).max() <= 5e-6 * np.abs(b).max()
    with pytest.raises(TypeError):
        overlap_batch(dm, px, py, mo, bloch, k0, s1_32, s2_32, precision='fp64')
