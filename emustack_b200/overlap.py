"""Bloch-mode / plane-wave overlap integrals and Bloch-mode normalisation on
the GPU (rows a11-a13 of the GSM stage).

``overlap_batch`` computes J (2 Npw x M) and J_dag (M x 2 Npw) for a batch of
wavelengths on one mesh (backend/fortran/J_overlap.f, J_dagger_overlap.f,
pw_ordering.f; J divided by the area ratio as backend/mode_calcs.py:384-386
does).  ``mode_normalisation`` computes the diagonal of the adjoint x prime
orthogonality matrix and the factors 1/sqrt(ovl)^2 that normalise the
adjoint modes (backend/fortran/orthogonal.f, normalisation.f).
``overlap_from_fields`` chains both for a drop-in ``Simmo``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import EmuNormalise, EmuOverlap, check, lib, ptr, stream_ptr

c128 = torch.complex128


class DeviceMesh(object):
    """A Mesh (emustack_b200.mesh) resident on the GPU."""

    def __init__(self, mesh, device='cuda'):
        self.mesh = mesh
        self.x, self.table_nod, self.type_el = mesh.to_device(device)
        self.nel, self.npt = mesh.nel, mesh.npt


def _dev_int32(a, dev):
    """Device int32 copy of an order list (kept as is if it already is one,
    so callers inside CUDA-graph capture make no host copies)."""
    if isinstance(a, torch.Tensor) and a.is_cuda and a.dtype == torch.int32:
        return a
    return torch.as_tensor(np.asarray(a, np.int32), device=dev)


def _check_sol(sol, nel, name, allow_c64=False):
    if sol is None:
        return
    ok = (torch.complex128, torch.complex64) if allow_c64 else (c128,)
    if sol.dtype not in ok or not sol.is_cuda or not sol.is_contiguous():
        raise TypeError('%s must be a contiguous CUDA %s tensor' % (
            name, 'complex128 or complex64' if allow_c64 else 'complex128'))
    if sol.dim() != 5 or tuple(sol.shape[1:2]) != (nel,) or tuple(sol.shape[3:]) != (13, 3):
        raise ValueError('%s must be [batch][nel][nval][13][3]' % name)


def overlap_batch(dmesh, px, py, max_order, bloch, k0, sol1=None, sol2=None, area_norm=1.0,
                  dy=1.0, scale2=None, perm2=None, elements_per_chunk=0, precision='fp64',
                  tc_splits=0, tune=True, check_error=True):
    """J, J_dag (device tensors) and index_pw_inv for a batch of problems.

    px, py     int32 [Npw] plane-wave orders (emustack_b200.films.grating_orders)
    bloch      float64 [B, 2] k_parallel * period;  k0 float64 [B] = 2 pi / wl_norm
    sol1/sol2  complex128 [B, nel, M, 13, 3] prime / adjoint fields (complex64
               accepted with precision='tf32x3': the operands are FP32 there,
               and the fields are read at half the bytes)
    scale2     complex128 [B, M] adjoint normalisation factors (or None)
    precision  'fp64' (FP64 GEMM) or 'tf32x3' (tensor cores, split-TF32 products)
    elements_per_chunk, tc_splits: launch choices (0 = defaults); with
               tune=True and both 0 the tensor-core path takes the
               autotuner's choice for this shape (timed on first use)
    check_error: read the tensor-core wait flag back (a host synchronisation);
               False inside CUDA-graph capture (the flag stays on the device)
    """
    dev = dmesh.x.device
    _check_sol(sol1, dmesh.nel, 'sol1', allow_c64=precision == 'tf32x3')
    _check_sol(sol2, dmesh.nel, 'sol2', allow_c64=precision == 'tf32x3')
    ref = sol1 if sol1 is not None else sol2
    c64 = ref.dtype == torch.complex64
    if sol1 is not None and sol2 is not None and sol1.dtype != sol2.dtype:
        raise TypeError('sol1 and sol2 must have the same dtype')
    B, M = int(ref.shape[0]), int(ref.shape[2])
    npw = len(px)
    d_px, d_py = _dev_int32(px, dev), _dev_int32(py, dev)
    for t, nm, dt in ((bloch, 'bloch', torch.float64), (k0, 'k0', torch.float64)):
        if t.dtype != dt or not t.is_cuda or not t.is_contiguous():
            raise TypeError('%s must be a contiguous CUDA %s tensor' % (nm, dt))
    J = torch.empty((B, 2 * npw, M), dtype=c128, device=dev) if sol1 is not None else None
    Jd = torch.empty((B, M, 2 * npw), dtype=c128, device=dev) if sol2 is not None else None
    inv = torch.empty((B, npw), dtype=torch.int32, device=dev)
    d = EmuOverlap()
    d.batch, d.nval, d.nel, d.npt = B, M, dmesh.nel, dmesh.npt
    d.n_pw, d.max_order = npw, int(max_order)
    d.d_px, d.d_py = ptr(d_px), ptr(d_py)
    d.d_x, d.d_table_nod = ptr(dmesh.x), ptr(dmesh.table_nod)
    d.d, d.dy = 1.0, float(dy)
    d.d_bloch, d.d_k0 = ptr(bloch), ptr(k0)
    d.d_sol1, d.d_sol2 = ptr(sol1), ptr(sol2)
    d.d_scale2, d.d_perm2 = ptr(scale2), ptr(perm2)
    d.area_norm = float(area_norm)
    d.d_J, d.d_J_dag, d.d_index_pw_inv = ptr(J), ptr(Jd), ptr(inv)
    d.elements_per_chunk = int(elements_per_chunk)
    if precision not in ('fp64', 'tf32x3'):
        raise ValueError("precision must be 'fp64' or 'tf32x3'")
    d.precision = 1 if precision == 'tf32x3' else 0
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    d.d_error = ptr(err)
    d.tc_splits = int(tc_splits)
    d.field_c64 = int(c64)
    L = lib()
    cands = None
    if d.precision == 1 and tune and not elements_per_chunk and not tc_splits:
        chunks = sorted({min(c, dmesh.nel) for c in (4096, 8192, 16384)})
        cands = [(c, 0) for c in chunks]
    sizes = []
    for c in (cands or [(d.elements_per_chunk, d.tc_splits)]):
        d.elements_per_chunk = c[0]
        sizes.append(L.emu_overlap_workspace_size(C.byref(d)))
    nbytes = max(sizes)
    ws = torch.empty(max(nbytes, 16), dtype=torch.uint8, device=dev)

    def run(c):
        d.elements_per_chunk, d.tc_splits = int(c[0]), int(c[1])
        check(L.emu_overlap_batch(C.byref(d), ptr(ws), C.c_size_t(nbytes), stream_ptr()),
              'emu_overlap_batch')

    choice = (int(elements_per_chunk), int(tc_splits))
    if cands:
        from .autotune import default_tuner, size_bucket
        shape = dict(npw=npw, M=M, nel=size_bucket(dmesh.nel), B=B, J=sol1 is not None,
                     Jd=sol2 is not None, c64=c64)
        choice = default_tuner().choose('overlap_tc', shape, cands, run, (0, 0))
    run(choice)
    if check_error and d.precision == 1 and int(err.item()) != 0:
        raise _lib.EmuError(6, 'emu_overlap_batch (tensor-core wait)')
    return J, Jd, inv


def tc_gemm(A, B, splits=4):
    """C = A B^T (float64 CUDA tensors [m, k], [n, k]) on the tensor cores
    with split-TF32 products (emu_tc_gemm_tf32x3)."""
    for t, nm in ((A, 'A'), (B, 'B')):
        if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous() or t.dim() != 2:
            raise TypeError('%s must be a contiguous CUDA float64 matrix' % nm)
    m, k = A.shape
    n = B.shape[0]
    if B.shape[1] != k:
        raise ValueError('inner dimensions differ')
    Cm = torch.empty((m, n), dtype=torch.float64, device=A.device)
    err = torch.zeros(1, dtype=torch.int32, device=A.device)
    L = lib()
    nbytes = L.emu_tc_gemm_workspace_size(m, n, k, splits)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=A.device)
    check(L.emu_tc_gemm_tf32x3(m, n, k, ptr(A), ptr(B), ptr(Cm), splits, ptr(err), ptr(ws),
                               C.c_size_t(nbytes), stream_ptr()), 'emu_tc_gemm_tf32x3')
    if int(err.item()) != 0:
        raise _lib.EmuError(6, 'emu_tc_gemm_tf32x3 (bounded wait)')
    return Cm


def mode_normalisation(dmesh, pp, k0, beta1, sol1, sol2):
    """Diagonal of the orthogonality matrix, normalisation factors and the
    count of |diag| <= 1e-7 per problem (device tensors)."""
    dev = dmesh.x.device
    _check_sol(sol1, dmesh.nel, 'sol1')
    _check_sol(sol2, dmesh.nel, 'sol2')
    B, M = int(sol1.shape[0]), int(sol1.shape[2])
    if not (isinstance(pp, torch.Tensor) and pp.is_cuda and pp.dtype == c128):
        pp = torch.as_tensor(np.asarray(pp, np.complex128), device=dev)
    if beta1.dtype != c128 or not beta1.is_cuda:
        raise TypeError('beta1 must be a CUDA complex128 tensor')
    if k0.dtype != torch.float64 or not k0.is_cuda or tuple(k0.shape) != (B,):
        raise TypeError('k0 must be a CUDA float64 tensor [batch]')
    diag = torch.empty((B, M), dtype=c128, device=dev)
    scale = torch.empty((B, M), dtype=c128, device=dev)
    nsmall = torch.empty((B,), dtype=torch.int32, device=dev)
    d = EmuNormalise()
    d.batch, d.nval, d.nel, d.npt = B, M, dmesh.nel, dmesh.npt
    d.d_x, d.d_table_nod, d.d_type_el = ptr(dmesh.x), ptr(dmesh.table_nod), ptr(dmesh.type_el)
    d.d_pp, d.d_k0, d.d_beta1 = ptr(pp), ptr(k0), ptr(beta1.contiguous())
    d.d_sol1, d.d_sol2 = ptr(sol1), ptr(sol2)
    d.d_diag, d.d_scale, d.d_n_small = ptr(diag), ptr(scale), ptr(nsmall)
    L = lib()
    nbytes = L.emu_mode_overlap_workspace_size(C.byref(d))
    ws = torch.empty(max(nbytes, 16), dtype=torch.uint8, device=dev)
    check(L.emu_mode_overlap_diag(C.byref(d), ptr(ws), C.c_size_t(nbytes), stream_ptr()),
          'emu_mode_overlap_diag')
    return diag, scale, nsmall


def mode_reorder(dmesh, pp, k0, beta1, sol1, sol2):
    """Conjugate-pair reordering of the adjoint modes (orthogonal.f:252-301)
    on the GPU: returns (perm, diag, scale, warn) device tensors; perm[b][i]
    is the adjoint mode at position i after the swaps."""
    dev = dmesh.x.device
    _check_sol(sol1, dmesh.nel, 'sol1')
    _check_sol(sol2, dmesh.nel, 'sol2')
    B, M = int(sol1.shape[0]), int(sol1.shape[2])
    pp = torch.as_tensor(np.asarray(pp, np.complex128), device=dev)
    if k0.dtype != torch.float64 or beta1.dtype != c128:
        raise TypeError('k0 must be float64 and beta1 complex128')
    diag = torch.empty((B, M), dtype=c128, device=dev)
    scale = torch.empty((B, M), dtype=c128, device=dev)
    perm = torch.empty((B, M), dtype=torch.int32, device=dev)
    warn = torch.empty((B,), dtype=torch.int32, device=dev)
    nsmall = torch.empty((B,), dtype=torch.int32, device=dev)
    d = EmuNormalise()
    d.batch, d.nval, d.nel, d.npt = B, M, dmesh.nel, dmesh.npt
    d.d_x, d.d_table_nod, d.d_type_el = ptr(dmesh.x), ptr(dmesh.table_nod), ptr(dmesh.type_el)
    d.d_pp, d.d_k0, d.d_beta1 = ptr(pp), ptr(k0), ptr(beta1.contiguous())
    d.d_sol1, d.d_sol2 = ptr(sol1), ptr(sol2)
    d.d_diag, d.d_scale, d.d_n_small = ptr(diag), ptr(scale), ptr(nsmall)
    L = lib()
    nbytes = L.emu_mode_overlap_reorder_workspace_size(C.byref(d))
    ws = torch.empty(max(nbytes, 16), dtype=torch.uint8, device=dev)
    check(L.emu_mode_overlap_reorder(C.byref(d), ptr(perm), ptr(warn), ptr(ws), C.c_size_t(nbytes),
                                     stream_ptr()), 'emu_mode_overlap_reorder')
    return perm, diag, scale, warn


def _on_device(a, dev):
    """complex128 contiguous tensor on ``dev`` from a numpy array or tensor."""
    if isinstance(a, torch.Tensor):
        return a.to(device=dev, dtype=torch.complex128).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a, np.complex128), device=dev)


def overlap_from_fields(simmo, fields):
    """J / area_norm and J_dag of a Simmo from its P2 mode fields.

    fields: dict with 'sol1', 'sol2' ([nel][M][13][3], the reference layout
    of sol(3, 13, M, nel)), 'beta1' (prime propagation constants; default
    simmo.k_z), 'pp' (per material type; default 1, the E-field
    formulation) and optionally 'mesh' (else simmo.structure.mesh).
    The adjoint modes are normalised on the GPU first.
    """
    from .films import grating_orders
    st = simmo.structure
    mesh = fields.get('mesh', getattr(st, 'mesh', None))
    if mesh is None:
        raise ValueError('overlap integrals need the mesh of the mode fields')
    dev = torch.device('cuda', torch.cuda.current_device())
    dm = fields.get('_device_mesh') or DeviceMesh(mesh, dev)
    sol1 = _on_device(fields['sol1'], dev).unsqueeze(0)
    sol2 = _on_device(fields['sol2'], dev).unsqueeze(0)
    M = sol1.shape[2]
    beta1 = torch.as_tensor(np.asarray(fields.get('beta1', simmo.k_z), np.complex128).reshape(1, M), device=dev)
    n_types = int(mesh.type_el.max())
    pp = fields.get('pp', np.ones(n_types, np.complex128))
    wl_norm = simmo.wl_norm()
    k0 = torch.tensor([2 * np.pi / wl_norm], dtype=torch.float64, device=dev)
    bloch = torch.tensor(np.asarray(simmo.k_pll_norm(), np.float64).reshape(1, 2), device=dev)
    diag, scale, nsmall = mode_normalisation(dm, pp, k0, beta1, sol1, sol2)
    perm = None
    if int(nsmall[0].item()) != 0:
        # a vanishing <m|m>: the reference reorders conjugate pairs first
        perm, diag, scale, warn = mode_reorder(dm, pp, k0, beta1, sol1, sol2)
        if int(warn[0].item()) != 0 and M <= 20:
            print('Warning found 1 BM of cmplx conj pair, increase num_BMs to include the other.')
    mo = simmo.max_order_PWs
    px, py = grating_orders(mo, st.period, st.period_y, False)
    area_norm = st.period_y / st.period
    J, Jd, inv = overlap_batch(dm, px, py, mo, bloch, k0, sol1, sol2, area_norm=area_norm,
                               dy=st.period_y / st.period, scale2=scale, perm2=perm,
                               precision=fields.get('precision', 'fp64'))
    simmo.overlap_diag = diag[0].cpu().numpy()
    return np.asmatrix(J[0].cpu().numpy()), np.asmatrix(Jd[0].cpu().numpy())


# ---------------------------------------------------------------------------
# 1D gratings (periodicity '1D_array')
# ---------------------------------------------------------------------------

class DeviceMesh1D(object):
    """A Mesh1D (emustack_b200.mesh) resident on the GPU."""

    def __init__(self, mesh, device='cuda'):
        self.mesh = mesh
        self.x = torch.tensor(mesh.x, device=device)
        self.table_nod = torch.tensor(mesh.table_nod, device=device)
        self.type_el = torch.tensor(mesh.type_el, device=device)
        self.nel, self.npt = mesh.nel, mesh.npt
        self.period_x = mesh.period_x


def pw_order_1d(max_order, period_x, bloch_x, bloch_y, k0):
    """0-based sorted position of each 1D order px = -max_order..max_order
    (emu_pw_order_1d: the reference's pw_ordering_1d ranking)."""
    out = np.empty(2 * max_order + 1, np.int32)
    check(lib().emu_pw_order_1d(int(max_order), float(period_x), float(bloch_x), float(bloch_y),
                                float(k0), out.ctypes.data_as(C.c_void_p)), 'emu_pw_order_1d')
    return out


def pw_rows_2d(max_order, period_x, bloch_x, bloch_y, k0):
    """(row of each 1D order in the sorted 2D order set, size of that set)
    (emu_pw_embed_1d_to_2d: the placement of pw_matrix_1d_to_2d)."""
    n = C.c_int(0)
    rows = np.empty(2 * max_order + 1, np.int32)
    check(lib().emu_pw_embed_1d_to_2d(int(max_order), float(period_x), float(bloch_x), float(bloch_y),
                                      float(k0), rows.ctypes.data_as(C.c_void_p), len(rows),
                                      C.byref(n)), 'emu_pw_embed_1d_to_2d')
    return rows, int(n.value)


def _check_sol1d(sol, nel, name):
    if sol is None:
        return
    if sol.dtype != c128 or not sol.is_cuda or not sol.is_contiguous():
        raise TypeError('%s must be a contiguous CUDA complex128 tensor' % name)
    if sol.dim() != 4 or sol.shape[1] != nel or sol.shape[3] != 11:
        raise ValueError('%s must be [batch][nel][nval][11]' % name)


def mode_overlap_1d(dmesh, pp, k0, bloch, beta1, sol1, sol2, perm2=None, full=False):
    """Orthogonality of adjoint and prime 1D modes (emu_mode_overlap_1d).
    full=False: (diag [B, M], scale [B, M], n_small [B]); full=True: the
    matrix [B, M, M]."""
    _check_sol1d(sol1, dmesh.nel, 'sol1')
    _check_sol1d(sol2, dmesh.nel, 'sol2')
    B, _, M, _ = sol1.shape
    dev = sol1.device
    for t, nm, dt, shape in ((k0, 'k0', torch.float64, (B,)), (bloch, 'bloch', torch.float64, (B, 2)),
                             (beta1, 'beta1', c128, (B, M))):
        if t.dtype != dt or not t.is_cuda or not t.is_contiguous() or tuple(t.shape) != shape:
            raise TypeError('%s must be a contiguous CUDA %s tensor of shape %s' % (nm, dt, shape))
    if perm2 is not None and (perm2.dtype != torch.int32 or tuple(perm2.shape) != (B, M)):
        raise TypeError('perm2 must be an int32 CUDA tensor [B, M]')
    pp_t = torch.as_tensor(np.asarray(pp, np.complex128), device=dev)
    d = _lib.EmuNormalise1D()
    d.batch, d.nval, d.nel, d.npt = B, M, dmesh.nel, dmesh.npt
    d.n_types = int(pp_t.numel())
    d.d_x, d.d_table_nod, d.d_type_el = ptr(dmesh.x), ptr(dmesh.table_nod), ptr(dmesh.type_el)
    d.d_pp, d.d_k0, d.d_bloch, d.d_beta1 = ptr(pp_t), ptr(k0), ptr(bloch), ptr(beta1)
    d.d_sol1, d.d_sol2 = ptr(sol1), ptr(sol2)
    d.d_perm2 = ptr(perm2)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    d.d_error = ptr(err)
    if full:
        out = torch.empty((B, M, M), dtype=c128, device=dev)
        d.d_out = ptr(out)
        check(lib().emu_mode_overlap_1d(C.byref(d), 1, stream_ptr()), 'emu_mode_overlap_1d')
        res = out
    else:
        diag = torch.empty((B, M), dtype=c128, device=dev)
        scale = torch.empty((B, M), dtype=c128, device=dev)
        nsmall = torch.zeros(B, dtype=torch.int32, device=dev)
        d.d_out, d.d_scale, d.d_n_small = ptr(diag), ptr(scale), ptr(nsmall)
        check(lib().emu_mode_overlap_1d(C.byref(d), 0, stream_ptr()), 'emu_mode_overlap_1d')
        res = (diag, scale, nsmall)
    if int(err.item()) != 0:
        raise ValueError('1D mesh: element nodes or material types out of range')
    return res


def reorder_pairs_1d(ovl):
    """Conjugate-pair swaps of the adjoint modes over the orthogonality
    matrix ``ovl`` [M, M] (rows adjoint, columns prime), as the loop of
    orthogonal_1d.f:160-215 performs them: a mode whose <j|j> vanishes
    (<= 1e-7) swaps its adjoint with every later adjoint j2 with
    |<j2|j>| > 1e-7, and the mode after it is left alone.  Returns the
    permutation (adjoint mode taken for each position) and the count of
    unpaired last modes (the reference's pair_warning)."""
    ovl = np.asarray(ovl)
    M = ovl.shape[0]
    perm = np.arange(M)
    warn = 0
    j, skip = 0, 0
    while j < M:
        if abs(ovl[j, j]) > 1e-7:
            j += 1
        elif skip == 0:
            if j == M - 1:
                warn += 1
            for j2 in range(j + 1, M):
                if abs(ovl[j2, j]) > 1e-7:
                    perm[j], perm[j2] = perm[j2], perm[j]
            skip = 1
            j += 1
        else:
            skip = 0
            j += 1
    return perm.astype(np.int32), warn


def overlap_1d_batch(dmesh, max_order, bloch, k0, sol1=None, sol2=None, scale=None, perm2=None,
                     embed_2d=False, period_x=None):
    """J [B, 2 Npw, M] and J_dag [B, M, 2 Npw] of 1D Bloch-mode fields
    (emu_overlap1d_batch), rows at the reference's sorted positions; with
    embed_2d also J_2d, J_dag_2d in the 2D order set.  bloch float64
    [B, 2] (k_parallel * period), k0 [B] (2 pi / wl_norm) as host arrays.
    Returns (J, J_dag, J_2d, J_dag_2d, index_pw_inv, rows_2d)."""
    _check_sol1d(sol1, dmesh.nel, 'sol1')
    _check_sol1d(sol2, dmesh.nel, 'sol2')
    ref = sol1 if sol1 is not None else sol2
    B, _, M, _ = ref.shape
    dev = ref.device
    px_ = float(dmesh.period_x if period_x is None else period_x)
    bloch = np.asarray(bloch, np.float64).reshape(B, 2)
    k0 = np.asarray(k0, np.float64).reshape(B)
    npw = 2 * max_order + 1
    inv = np.stack([pw_order_1d(max_order, px_, bloch[b, 0], bloch[b, 1], k0[b]) for b in range(B)])
    rows = npw2 = None
    if embed_2d:
        r = [pw_rows_2d(max_order, px_, bloch[b, 0], bloch[b, 1], k0[b]) for b in range(B)]
        rows = np.stack([x[0] for x in r])
        npw2 = r[0][1]
    d = _lib.EmuOverlap1D()
    d.batch, d.nval, d.nel, d.npt, d.max_order = B, M, dmesh.nel, dmesh.npt, int(max_order)
    d.d_x, d.d_table_nod, d.period_x = ptr(dmesh.x), ptr(dmesh.table_nod), px_
    d_bloch = torch.tensor(bloch, device=dev)
    d_inv = torch.tensor(inv, dtype=torch.int32, device=dev)
    d.d_bloch, d.d_index_pw_inv = ptr(d_bloch), ptr(d_inv)
    d.d_sol1, d.d_sol2, d.d_scale, d.d_perm2 = ptr(sol1), ptr(sol2), ptr(scale), ptr(perm2)
    J = torch.empty((B, 2 * npw, M), dtype=c128, device=dev) if sol1 is not None else None
    Jd = torch.empty((B, M, 2 * npw), dtype=c128, device=dev) if sol2 is not None else None
    d.d_J, d.d_J_dag = ptr(J), ptr(Jd)
    J2 = Jd2 = d_rows = None
    if embed_2d:
        d.npw_2d = npw2
        d_rows = torch.tensor(rows, dtype=torch.int32, device=dev)
        d.d_row_2d = ptr(d_rows)
        if sol1 is not None:
            J2 = torch.empty((B, 2 * npw2, M), dtype=c128, device=dev)
        if sol2 is not None:
            Jd2 = torch.empty((B, M, 2 * npw2), dtype=c128, device=dev)
        d.d_J_2d, d.d_J_dag_2d = ptr(J2), ptr(Jd2)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    d.d_error = ptr(err)
    check(lib().emu_overlap1d_batch(C.byref(d), stream_ptr()), 'emu_overlap1d_batch')
    if int(err.item()) != 0:
        raise ValueError('1D mesh: element nodes out of range')
    return J, Jd, J2, Jd2, inv, rows


def overlap_from_fields_1d(simmo, fields):
    """J and J_dag of a 1D-grating Simmo from its mode fields, as
    backend/fortran/py_calc_modes_1d.f:525-620 and backend/mode_calcs.py:
    323-355 produce them: orthogonality of adjoint and prime modes, the
    conjugate-pair swaps, normalisation of both by 1/sqrt(<m|m>), then J,
    J_dag (in the 1D order set for world_1d layers, embedded in the 2D set
    otherwise; no area division for 1D layers).

    fields: 'sol1', 'sol2' ([nel][M][11], the reference layout of
    sol(11, M, nel)), 'beta1' (default simmo.k_z), 'pp' (per material type,
    default 1) and optionally 'mesh' (a Mesh1D, else simmo.structure.mesh).
    """
    st = simmo.structure
    mesh = fields.get('mesh', getattr(st, 'mesh', None))
    if mesh is None:
        raise ValueError('overlap integrals need the mesh of the mode fields')
    dev = torch.device('cuda', torch.cuda.current_device())
    dm = DeviceMesh1D(mesh, dev)
    sol1 = _on_device(fields['sol1'], dev).unsqueeze(0)
    sol2 = _on_device(fields['sol2'], dev).unsqueeze(0)
    M = sol1.shape[2]
    beta1 = torch.as_tensor(np.asarray(fields.get('beta1', simmo.k_z), np.complex128).reshape(1, M),
                            device=dev)
    pp = fields.get('pp', np.ones(int(mesh.type_el.max()), np.complex128))
    k0v = 2 * np.pi / simmo.wl_norm()
    bl = np.asarray(simmo.k_pll_norm(), np.float64).reshape(1, 2)
    k0 = torch.tensor([k0v], dtype=torch.float64, device=dev)
    bloch = torch.tensor(bl, device=dev)
    diag, scale, nsmall = mode_overlap_1d(dm, pp, k0, bloch, beta1, sol1, sol2)
    perm = None
    if int(nsmall[0].item()) != 0:
        full = mode_overlap_1d(dm, pp, k0, bloch, beta1, sol1, sol2, full=True)[0].cpu().numpy()
        p, warn = reorder_pairs_1d(full)
        if warn and M <= 20:
            print('Warning found 1 BM of cmplx conj pair, increase num_BMs to include the other.')
        perm = torch.tensor(p.reshape(1, M), device=dev)
        diag, scale, _ = mode_overlap_1d(dm, pp, k0, bloch, beta1, sol1, sol2, perm2=perm)
    w1d = bool(st.world_1d)
    J, Jd, J2, Jd2, _, _ = overlap_1d_batch(dm, simmo.max_order_PWs, bl, [k0v], sol1, sol2, scale=scale,
                                            perm2=perm, embed_2d=not w1d)
    simmo.overlap_diag = diag[0].cpu().numpy()
    if w1d:
        return np.asmatrix(J[0].cpu().numpy()), np.asmatrix(Jd[0].cpu().numpy())
    return np.asmatrix(J2[0].cpu().numpy()), np.asmatrix(Jd2[0].cpu().numpy())
