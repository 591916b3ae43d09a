"""FEM Bloch modes of 2D nanostructured layers on the GPU (the reference's
calc_modes_2d, backend/fortran/py_calc_modes.f:243-700, as
backend/mode_calcs.py:268-381 calls it: E-field formulation, periodic cell).

Per layer and Bloch vector:

1. element matrices K_e, M_e on the device (``emu_fem_element_matrices``),
   summed onto the CSR pattern in element order (``emu_fem_assemble``);
2. the shifted matrix A = K - shift M, dense on the device, factored by a
   blocked LU with FP64 tensor-core GEMM tiles (``emu_fem_lu``) and inverted
   (``emu_fem_inverse``), so that every application of the operator is one
   sparse product and one dense GEMM;
3. the nval eigenvalues of OP = A^-1 M of largest modulus by a block
   Krylov-Schur iteration (Stewart, SIAM J. Matrix Anal. Appl. 23, 2001, in
   block form): OP applied to blocks of ``block`` vectors at once
   (``emu_fem_apply_op``: sparse M times the block, non-zero only on the
   transverse DOFs, then the matching columns of A^-1 times that),
   the basis orthogonalised by two classical Gram-Schmidt passes and
   Cholesky QR on the device; the small projected matrix (at most
   ``max_basis`` square) is reduced to an ordered Schur form on the host and
   the basis restarted on its leading Schur vectors, as ARPACK's reverse-communication loop does
   its small dense steps on the host (valpr_umf_64.f:300-470 runs ARPACK's
   implicitly restarted Arnoldi with one vector per step);
4. beta^2 = 1/nu + shift with the reference's branch rule, the modes ranked by
   -Re(beta^2) with the reference's quicksort (``emu_fem_mode_order``), and
   the nodal fields of array_sol.f with its max-modulus normalisation
   (``emu_fem_nodal_fields``).

The dense factorisation is exact and simple but grows as neq^2 in memory and
neq^3 in work (two 16 neq^2-byte matrices: 1.2 GB at the reference's
518-element test mesh, 29 GB at 30 000 DOFs).
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np
import torch

from . import _lib
from ._lib import check, lib, ptr, stream_ptr


class FemMesh(object):
    """A P2 mesh of the unit cell with its DOF topology, resident on the GPU.

    ``x`` [npt][2] in units of the period, ``type_nod`` [npt] (non-zero on
    the cell boundary, the .mail files' node type), ``table_nod`` [nel][6]
    1-based, ``type_el`` [nel] 1-based material index."""

    def __init__(self, x, type_nod, table_nod, type_el, device=None):
        self.x = np.ascontiguousarray(x, np.float64)
        self.type_nod = np.ascontiguousarray(type_nod, np.int32)
        self.table_nod = np.ascontiguousarray(table_nod, np.int64)
        self.type_el = np.ascontiguousarray(type_el, np.int64)
        npt, nel = len(self.x), len(self.table_nod)
        self.npt, self.nel = npt, nel
        dof = np.zeros((nel, 22), np.int32)
        shift = np.zeros((nel, 14, 2), np.float64)
        ends = np.zeros((nel, 3, 2), np.int8)
        row_ptr = np.zeros(nel * 22 + 1, np.int32)
        col = np.zeros(nel * 484, np.int32)
        src_ptr = np.zeros(nel * 484 + 1, np.int32)
        src = np.zeros(nel * 484, np.int32)
        t = _lib.EmuFemTopology()
        t.npt, t.nel = npt, nel
        arrays = (self.x, self.type_nod, self.table_nod, dof, shift, ends, row_ptr, col, src_ptr, src)
        (t.h_x, t.h_type_nod, t.h_table_nod, t.h_dof, t.h_shift, t.h_ends, t.h_row_ptr, t.h_col,
         t.h_src_ptr, t.h_src) = [a.ctypes.data_as(C.c_void_p) for a in arrays]
        check(lib().emu_fem_topology(C.byref(t)), 'emu_fem_topology')
        self.neq, self.nnz = t.neq, t.nnz
        self.dof, self.shift, self.ends = dof, shift, ends
        dev = torch.device('cuda', torch.cuda.current_device()) if device is None else torch.device(device)
        self.device = dev
        up = lambda a: torch.as_tensor(np.ascontiguousarray(a)).to(dev)
        self.d_x, self.d_table_nod, self.d_type_el = up(self.x), up(self.table_nod), up(self.type_el)
        self.d_shift, self.d_ends, self.d_dof = up(shift), up(ends), up(dof)
        self.d_row_ptr = up(row_ptr[:self.neq + 1])
        self.d_col = up(col[:self.nnz])
        self.d_src_ptr = up(src_ptr[:self.nnz + 1])
        self.d_src = up(src)
        # rows where M has entries: the transverse DOFs (faces and edges)
        self.trows = np.unique(dof[:, :12]).astype(np.int32)
        self.d_trows = up(self.trows)

    @classmethod
    def from_mail(cls, path, device=None):
        """Read a .mail mesh (npt nel; npt rows 'k x y type'; nel rows 'k n1..n6 type')."""
        with open(path) as f:
            tok = f.read().split()
        npt, nel = int(tok[0]), int(tok[1])
        pts = np.array(tok[2:2 + 4 * npt], dtype=float).reshape(npt, 4)
        p = 2 + 4 * npt
        els = np.array(tok[p:p + 8 * nel], dtype=np.int64).reshape(nel, 8)
        return cls(pts[:, 1:3], pts[:, 3].astype(np.int32), els[:, 1:7], els[:, 7], device)

    @classmethod
    def from_mesh(cls, mesh, device=None):
        """From an emustack_b200.mesh.Mesh that carries its boundary node types."""
        if getattr(mesh, 'type_nod', None) is None:
            raise ValueError('the FEM solve needs the boundary node types of the mesh (Mesh.from_mail)')
        return cls(mesh.x, mesh.type_nod, mesh.table_nod, mesh.type_el, device)

    def element_matrices(self, n_effs, k0, bloch, s):
        """K_e, M_e [nel][22][22] on the device (emu_fem_element_matrices)."""
        n_effs = np.asarray(n_effs, np.complex128).ravel()
        n_types = int(self.type_el.max())
        if len(n_effs) < n_types or n_types > 8:
            raise ValueError('need the index of each of the mesh\'s %d material types' % n_types)
        Ke = torch.empty((self.nel, 22, 22), dtype=torch.complex128, device=self.device)
        Me = torch.empty_like(Ke)
        e = _lib.EmuFemElements()
        e.nel, e.n_types = self.nel, n_types
        e.d_x, e.d_table_nod, e.d_type_el = ptr(self.d_x), ptr(self.d_table_nod), ptr(self.d_type_el)
        e.d_shift, e.d_ends = ptr(self.d_shift), ptr(self.d_ends)
        for i in range(min(8, len(n_effs))):
            e.n_eff[i] = _c128(n_effs[i])
        e.k0 = float(k0)
        e.bloch[0], e.bloch[1] = float(bloch[0]), float(bloch[1])
        e.d_Ke, e.d_Me = ptr(Ke), ptr(Me)
        check(lib().emu_fem_element_matrices(C.byref(e), s), 'emu_fem_element_matrices')
        return Ke, Me

    def nodal_fields(self, Y, nval, bloch, adjoint, s):
        """sol [nel][nval][13][3] from eigenvectors Y [neq][nval] (emu_fem_nodal_fields)."""
        sol = torch.empty((self.nel, nval, 13, 3), dtype=torch.complex128, device=self.device)
        f = _lib.EmuFemFields()
        f.nel, f.neq, f.nval = self.nel, self.neq, nval
        f.d_x, f.d_table_nod, f.d_shift, f.d_ends, f.d_dof = (ptr(self.d_x), ptr(self.d_table_nod),
                                                              ptr(self.d_shift), ptr(self.d_ends), ptr(self.d_dof))
        f.bloch[0], f.bloch[1] = float(bloch[0]), float(bloch[1])
        f.d_vec, f.ldv, f.d_sol = ptr(Y), nval, ptr(sol)
        ws_bytes = lib().emu_fem_fields_workspace_size(C.byref(f))
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device=self.device)
        check(lib().emu_fem_nodal_fields(C.byref(f), ptr(ws), ws_bytes, s), 'emu_fem_nodal_fields')
        return sol


class FemMesh1D(object):
    """A 1D grating's P2 mesh with its DOF topology (emu_fem1d_topology),
    resident on the GPU.  ``x`` [npt] P2 node coordinates (any unit: the
    cell is rescaled to length 1, the unit of the normalised wavelength),
    ``table_nod`` [nel][3] 1-based (x_min node, x_max node, middle node),
    elements left to right, ``type_el`` [nel] 1-based material index."""

    def __init__(self, x, table_nod, type_el, device=None):
        x = np.ascontiguousarray(x, np.float64).ravel()
        self.table_nod = np.ascontiguousarray(table_nod, np.int64)
        if self.table_nod.ndim != 2 or self.table_nod.shape[1] != 3:
            raise ValueError('table_nod must be [nel][3]')
        self.type_el = np.ascontiguousarray(type_el, np.int64)
        nel = len(self.table_nod)
        x0 = x[self.table_nod[0, 0] - 1]
        span = x[self.table_nod[-1, 1] - 1] - x0
        self.x = (x - x0) / span if span > 0 else x
        self.npt, self.nel = len(x), nel
        dof = np.zeros((nel, 11), np.int32)
        shift = np.zeros((nel, 11), np.float64)
        row_ptr = np.zeros(9 * nel + 1, np.int32)
        col = np.zeros(121 * nel, np.int32)
        src_ptr = np.zeros(121 * nel + 1, np.int32)
        src = np.zeros(121 * nel, np.int32)
        t = _lib.EmuFem1dTopology()
        t.npt, t.nel = self.npt, nel
        arrays = (self.x, self.table_nod, dof, shift, row_ptr, col, src_ptr, src)
        (t.h_x, t.h_table_nod, t.h_dof, t.h_shift, t.h_row_ptr, t.h_col, t.h_src_ptr,
         t.h_src) = [a.ctypes.data_as(C.c_void_p) for a in arrays]
        check(lib().emu_fem1d_topology(C.byref(t)), 'emu_fem1d_topology')
        self.neq, self.nnz = t.neq, t.nnz
        self.dof, self.shift = dof, shift
        dev = torch.device('cuda', torch.cuda.current_device()) if device is None else torch.device(device)
        self.device = dev
        up = lambda a: torch.as_tensor(np.ascontiguousarray(a)).to(dev)
        self.d_x, self.d_table_nod, self.d_type_el = up(self.x), up(self.table_nod), up(self.type_el)
        self.d_shift, self.d_dof = up(shift), up(dof)
        self.d_row_ptr = up(row_ptr[:self.neq + 1])
        self.d_col = up(col[:self.nnz])
        self.d_src_ptr = up(src_ptr[:self.nnz + 1])
        self.d_src = up(src)
        # rows where M has entries: the E_x and E_y DOFs
        self.trows = np.unique(dof[:, :7]).astype(np.int32)
        self.d_trows = up(self.trows)

    @classmethod
    def from_mesh(cls, mesh, device=None):
        """From an emustack_b200.mesh.Mesh1D."""
        return cls(mesh.x, mesh.table_nod, mesh.type_el, device)

    def element_matrices(self, n_effs, k0, bloch, s):
        """K_e, M_e [nel][11][11] on the device (emu_fem1d_element_matrices)."""
        n_effs = np.asarray(n_effs, np.complex128).ravel()
        n_types = int(self.type_el.max())
        if len(n_effs) < n_types or n_types > 8:
            raise ValueError('need the index of each of the mesh\'s %d material types' % n_types)
        Ke = torch.empty((self.nel, 11, 11), dtype=torch.complex128, device=self.device)
        Me = torch.empty_like(Ke)
        e = _lib.EmuFem1dElements()
        e.nel, e.n_types = self.nel, n_types
        e.d_x, e.d_table_nod, e.d_type_el, e.d_shift = (ptr(self.d_x), ptr(self.d_table_nod),
                                                        ptr(self.d_type_el), ptr(self.d_shift))
        for i in range(min(8, len(n_effs))):
            e.n_eff[i] = _c128(n_effs[i])
        e.k0 = float(k0)
        e.bloch[0], e.bloch[1] = float(bloch[0]), float(bloch[1])
        e.d_Ke, e.d_Me = ptr(Ke), ptr(Me)
        check(lib().emu_fem1d_element_matrices(C.byref(e), s), 'emu_fem1d_element_matrices')
        return Ke, Me

    def nodal_fields(self, Y, nval, bloch, adjoint, s):
        """sol [nel][nval][11] from eigenvectors Y [neq][nval] (emu_fem1d_nodal_fields)."""
        sol = torch.empty((self.nel, nval, 11), dtype=torch.complex128, device=self.device)
        f = _lib.EmuFem1dFields()
        f.nel, f.neq, f.nval = self.nel, self.neq, nval
        f.d_x, f.d_table_nod, f.d_shift, f.d_dof = (ptr(self.d_x), ptr(self.d_table_nod), ptr(self.d_shift),
                                                    ptr(self.d_dof))
        f.bloch_x, f.adjoint = float(bloch[0]), int(bool(adjoint))
        f.d_vec, f.ldv, f.d_sol = ptr(Y), nval, ptr(sol)
        ws_bytes = lib().emu_fem1d_fields_workspace_size(C.byref(f))
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device=self.device)
        check(lib().emu_fem1d_nodal_fields(C.byref(f), ptr(ws), ws_bytes, s), 'emu_fem1d_nodal_fields')
        return sol


def _c128(z):
    z = complex(z)
    return _lib.EmuC128(z.real, z.imag)


def shift_of(n_effs, k0, bloch):
    """The shift-and-invert centre of backend/mode_calcs.py:300-310 (not
    hyperbolic): 1.1 max(Re n)^2 k0^2 - |k_parallel|^2."""
    return 1.1 * np.real(np.asarray(n_effs)).max() ** 2 * k0 ** 2 - bloch[0] ** 2 - bloch[1] ** 2


def beta_branch(b2):
    """sqrt(beta^2) with the branch of py_calc_modes.f:664-674."""
    b = np.sqrt(np.asarray(b2, complex))
    flip = np.where(np.abs(b.imag) < 1e-8, b.real < 0, b.imag < 0)
    return np.where(flip, -b, b)


class _NoLimit(object):
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def _one_blas_thread():
    """A context that limits the host BLAS / LAPACK to one thread
    (threadpoolctl; a no-op where it is absent)."""
    try:
        from threadpoolctl import threadpool_limits
        return threadpool_limits(limits=1)
    except Exception:
        return _NoLimit()


_LINALG_READY = set()


def _linalg_ready(dev):
    """Run torch's device linear-algebra entry points once in this thread:
    their first call initialises a library handle, which two threads must not
    do at once."""
    if dev in _LINALG_READY:
        return
    G = torch.eye(2, dtype=torch.complex128, device=dev)
    L, _ = torch.linalg.cholesky_ex(G)
    torch.linalg.solve_triangular(L.conj().T, G, upper=True, left=False)
    torch.cuda.synchronize(dev)
    _LINALG_READY.add(dev)


def mode_order(beta):
    """0-based order of the modes by -Re(beta^2), the reference's quicksort."""
    beta = np.ascontiguousarray(beta, np.complex128)
    idx = np.zeros(len(beta), np.int32)
    check(lib().emu_fem_mode_order(len(beta), beta.ctypes.data_as(C.c_void_p), idx.ctypes.data_as(C.c_void_p)),
          'emu_fem_mode_order')
    return idx


class FemModeSolver(object):
    """Shift-and-invert mode solve of one mesh (see the module docstring).

    block: vectors per application of OP; max_basis: Krylov basis size before
    a restart; keep: Schur vectors kept at a restart; tol: residual
    |OP y - nu y| / |nu| of the wanted Ritz pairs.

    The defaults (4 vectors per application, a basis of max(2.5 nval, nval +
    20 blocks), nval + nval / 2 kept) trade more applications of the operator
    for fewer and smaller Schur forms on the host, which cost more than the
    operator's pass over A^-1: on the reference's 2D test mesh (6 216 DOFs,
    40 modes) one layer takes 0.58 s against 0.96-0.99 s with blocks of 16
    and a basis of 176, on its 1D gratings (1 800 DOFs, 46 modes) 0.11-0.12 s
    against 0.25-0.40 s."""

    def __init__(self, mesh, block=4, max_basis=None, keep=None, tol=1e-13, max_restarts=200, seed=20261204):
        self.mesh = mesh
        self.block, self.max_basis, self.keep = block, max_basis, keep
        self.tol, self.max_restarts, self.seed = tol, max_restarts, seed
        self.stats = {}

    # -- operator -------------------------------------------------------
    def factor(self, n_effs, k0, bloch, shift, stream=None):
        """Assemble K, M for this Bloch vector and factor K - shift M."""
        m = self.mesh
        dev = m.device
        s = stream_ptr(stream)
        Ke, Me = m.element_matrices(n_effs, k0, bloch, s)
        self.K = torch.empty(m.nnz, dtype=torch.complex128, device=dev)
        self.M = torch.empty_like(self.K)
        check(lib().emu_fem_assemble(m.nnz, ptr(m.d_src_ptr), ptr(m.d_src), ptr(Ke), ptr(Me), ptr(self.K),
                                     ptr(self.M), s), 'emu_fem_assemble')
        del Ke, Me
        n = m.neq
        self.A = torch.empty((n, n), dtype=torch.complex128, device=dev)
        check(lib().emu_fem_shifted_dense(n, ptr(m.d_row_ptr), ptr(m.d_col), ptr(self.K), ptr(self.M),
                                          _c128(shift), ptr(self.A), n, s), 'emu_fem_shifted_dense')
        self.ipiv = torch.empty(n, dtype=torch.int32, device=dev)
        info = torch.zeros(1, dtype=torch.int32, device=dev)
        check(lib().emu_fem_lu(n, ptr(self.A), n, ptr(self.ipiv), ptr(info), s), 'emu_fem_lu')
        if int(info.item()) != 0:
            raise _lib.EmuError(_lib.EMU_E_SINGULAR, 'emu_fem_lu (K - shift M is singular)')
        nt = len(m.trows)
        self.Ainv = torch.empty((n, nt), dtype=torch.complex128, device=dev)
        check(lib().emu_fem_inverse(n, ptr(self.A), n, ptr(self.ipiv), nt, ptr(m.d_trows), ptr(self.Ainv), nt, s),
              'emu_fem_inverse')
        del self.A

    def apply(self, X, Y, stream=None):
        """Y = (K - shift M)^-1 M X for a column block X of a row-major
        [n][ld] tensor (X and Y may be strided views with unit column stride)."""
        m = self.mesh
        n, nt = m.neq, len(m.trows)
        nrhs = X.shape[1]
        T = getattr(self, '_T', None)
        if T is None or T.numel() < nt * nrhs:
            T = self._T = torch.empty(nt * nrhs, dtype=torch.complex128, device=X.device)
        check(lib().emu_fem_apply_op(n, nrhs, ptr(self.Ainv), nt, nt, ptr(m.d_trows), ptr(m.d_row_ptr),
                                     ptr(m.d_col), ptr(self.M), ptr(X), X.stride(0), ptr(T), ptr(Y), Y.stride(0),
                                     stream_ptr(stream)), 'emu_fem_apply_op')

    # -- block Krylov-Schur ---------------------------------------------
    @staticmethod
    def _cholqr(W):
        """W = Q R with Q orthonormal (two Cholesky QR passes); returns
        (Q, R) or (None, None) when W is numerically rank deficient."""
        Rt = None
        for _ in range(2):
            G = W.conj().T @ W
            L, info = torch.linalg.cholesky_ex(G)
            if int(info.item()) != 0:
                return None, None
            R = L.conj().T
            W = torch.linalg.solve_triangular(R, W, upper=True, left=False)
            Rt = R if Rt is None else R @ Rt
        return W, Rt

    def eigs(self, nval, stream=None):
        """The nval eigenpairs of OP of largest |nu|: (nu [nval] numpy,
        eigenvectors [n][nval] device tensor)."""
        import scipy.linalg as sl
        from scipy.linalg import lapack
        n = self.mesh.neq
        dev = self.mesh.device
        b = min(self.block, n)
        mmax = self.max_basis or max(2 * nval + nval // 2 + 3, nval + 20 * b)
        mmax = int(min(-(-mmax // b) * b, n - b))
        keep = self.keep or min(mmax - b, nval + max(b, nval // 2))
        if nval + 1 > keep or keep + b > mmax:
            raise ValueError('basis too small for %d modes (n = %d)' % (nval, n))
        gen = torch.Generator(device='cpu').manual_seed(self.seed)
        V = torch.zeros((n, mmax + b), dtype=torch.complex128, device=dev)
        X0 = torch.complex(torch.randn(n, b, generator=gen, dtype=torch.float64),
                           torch.randn(n, b, generator=gen, dtype=torch.float64)).to(dev)
        Q0, _ = self._cholqr(X0)
        V[:, :b] = Q0
        H = np.zeros((mmax + b, mmax), complex)
        W = torch.empty((n, b), dtype=torch.complex128, device=dev)
        m = 0
        applies = 0
        host_s = 0.0
        for restart in range(self.max_restarts):
            while m + b <= mmax:
                self.apply(V[:, m:m + b], W, stream)
                applies += 1
                Vm = V[:, :m + b]
                Cc = Vm.conj().T @ W
                W -= Vm @ Cc
                C2 = Vm.conj().T @ W
                W -= Vm @ C2
                Cc += C2
                # two Cholesky QR passes; one device-to-host copy per step
                L1, i1 = torch.linalg.cholesky_ex(W.conj().T @ W)
                R1 = L1.conj().T
                W1 = torch.linalg.solve_triangular(R1, W, upper=True, left=False)
                L2, i2 = torch.linalg.cholesky_ex(W1.conj().T @ W1)
                R2 = L2.conj().T
                Q = torch.linalg.solve_triangular(R2, W1, upper=True, left=False)
                R = R2 @ R1
                host = torch.cat([Cc.reshape(-1), R.reshape(-1),
                                  (i1 + i2).to(torch.complex128).reshape(-1)]).cpu().numpy()
                Ch = host[:(m + b) * b].reshape(m + b, b)
                Rh = host[(m + b) * b:(m + b) * b + b * b].reshape(b, b)
                if host[-1].real != 0 or not np.all(np.isfinite(Rh)):
                    # the Krylov space closed: continue with fresh directions
                    Xr = torch.complex(torch.randn(n, b, generator=gen, dtype=torch.float64),
                                       torch.randn(n, b, generator=gen, dtype=torch.float64)).to(dev)
                    Xr -= Vm @ (Vm.conj().T @ Xr)
                    Xr -= Vm @ (Vm.conj().T @ Xr)
                    Q, _ = self._cholqr(Xr)
                    Rh = np.zeros((b, b), complex)
                H[:m + b, m:m + b] = Ch
                H[m + b:m + 2 * b, m:m + b] = Rh
                V[:, m + b:m + 2 * b] = Q
                m += b
            t_host = time.perf_counter()
            Hm = H[:m, :m]
            # the projected matrix is small: one host thread reduces it as fast as
            # many, and two solves running side by side then do not oversubscribe
            with _one_blas_thread():
                # Krylov-Schur restart (Stewart 2001): a unitary Schur form of the
                # projected matrix, reordered so that the wanted Ritz values lead;
                # the kept basis V Q_k and block T_k keep the Krylov relation exact
                T, Q = sl.schur(Hm, output='complex')
                ev = np.diag(T)
                order = np.argsort(-np.abs(ev), kind='stable')
                sel = np.zeros(m, np.int32)
                sel[order[:nval]] = 1
                Tw, Qw = lapack.ztrsen(sel, T, Q, job='N')[:2]
                th, Wv = np.linalg.eig(Tw[:nval, :nval])
                o = np.argsort(-np.abs(th), kind='stable')
                th, Wv = th[o], Wv[:, o]
                Z = Qw[:, :nval] @ Wv
                Z /= np.linalg.norm(Z, axis=0)
                res = np.linalg.norm(H[m:m + b, :m] @ Z, axis=0) / np.abs(th)
            if res.max() < self.tol:
                Zd = torch.as_tensor(np.ascontiguousarray(Z)).to(dev)
                Y = V[:, :m] @ Zd
                host_s += time.perf_counter() - t_host
                self.stats = {'applies': applies, 'restarts': restart, 'basis': mmax, 'block': b,
                              'residual': float(res.max()), 'host_projection_s': host_s}
                return th, Y
            k = int(min(keep, mmax - b))
            sel = np.zeros(m, np.int32)
            sel[order[:k]] = 1
            with _one_blas_thread():
                Tk, Qk_h = lapack.ztrsen(sel, T, Q, job='N')[:2]
            Qk = torch.as_tensor(np.ascontiguousarray(Qk_h[:, :k])).to(dev)
            tail = V[:, m:m + b].clone()
            V[:, :k] = V[:, :m] @ Qk
            V[:, k:k + b] = tail
            Hn = np.zeros_like(H)
            Hn[:k, :k] = np.triu(Tk[:k, :k])
            Hn[k:k + b, :k] = H[m:m + b, :m] @ Qk_h[:, :k]
            H = Hn
            m = k
            host_s += time.perf_counter() - t_host
        raise RuntimeError('FEM eigen-solve: no convergence in %d restarts (residual %.1e)'
                           % (self.max_restarts, res.max()))

    # -- the solve of calc_modes_2d -------------------------------------
    def solve(self, n_effs, wl_norm, bloch, nval, shift=None, stream=None, adjoint=False):
        """beta [nval] (numpy, sorted) and the nodal fields (device; 2D:
        [nel][nval][13][3], 1D: [nel][nval][11]) for the Bloch vector
        ``bloch`` (k_parallel * period); ``adjoint`` marks the solve of the
        adjoint modes (the 1D normalisation differs for them)."""
        k0 = 2 * np.pi / wl_norm
        bloch = np.asarray(bloch, np.float64)
        if shift is None:
            shift = shift_of(n_effs, k0, bloch)
        self.factor(n_effs, k0, bloch, shift, stream)
        nu, Y = self.eigs(nval, stream)
        del self.Ainv
        beta = beta_branch(1.0 / nu + shift)
        order = mode_order(beta)
        beta = beta[order]
        Y = Y[:, torch.as_tensor(order.astype(np.int64)).to(Y.device)].contiguous()
        sol = self.mesh.nodal_fields(Y, nval, bloch, adjoint, stream_ptr(stream))
        return beta, sol

    def solve_pair(self, n_effs, wl_norm, bloch, nval, shift=None, stream=None, concurrent=True):
        """The prime modes (Bloch vector ``bloch``) and the adjoint modes
        (-bloch) as calc_modes_2d solves both (py_calc_modes.f:604-616):
        beta1, sol1, beta2, sol2.  ``concurrent``: the two solves run on two
        streams from two host threads, so that one solve's host steps (the
        projected eigenproblems) overlap the other's device work."""
        bloch = np.asarray(bloch, np.float64)
        if not concurrent:
            b1, s1 = self.solve(n_effs, wl_norm, bloch, nval, shift, stream)
            b2, s2 = self.solve(n_effs, wl_norm, -bloch, nval, shift, stream, adjoint=True)
            return b1, s1, b2, s2
        import threading
        _linalg_ready(self.mesh.device)
        other = FemModeSolver(self.mesh, block=self.block, max_basis=self.max_basis, keep=self.keep,
                              tol=self.tol, max_restarts=self.max_restarts, seed=self.seed)
        caller = stream if stream is not None else torch.cuda.current_stream()
        streams = (torch.cuda.Stream(), torch.cuda.Stream())
        for st in streams:
            st.wait_stream(caller)
        out, errs = [None, None], []

        def run(i, solver, b):
            try:
                with torch.cuda.stream(streams[i]):
                    out[i] = solver.solve(n_effs, wl_norm, b, nval, shift, streams[i], adjoint=i == 1)
            except BaseException as e:  # re-raised in the calling thread
                errs.append(e)

        t = threading.Thread(target=run, args=(1, other, -bloch))
        t.start()
        run(0, self, bloch)
        t.join()
        for st in streams:
            caller.wait_stream(st)
        if errs:
            raise errs[0]
        self.stats_adjoint = other.stats
        return out[0][0], out[0][1], out[1][0], out[1][1]


def solve_pairs(mesh, jobs, nval, workers=4, **solver_args):
    """Prime and adjoint modes of one mesh for many (n_effs, wl_norm, bloch,
    shift) jobs (a wavelength sweep, as the reference maps calc_modes over
    wavelengths with a process pool): ``workers`` host threads, each with its
    own solver and stream, so that one job's host steps overlap the others'
    device work.  Returns [(beta1, sol1, beta2, sol2)] in the order of
    ``jobs``; the results agree with those of solving the jobs one by one to
    the solver's accuracy (cuBLAS's reductions in the Krylov basis may round
    differently while several streams run)."""
    import concurrent.futures as cf
    import threading
    jobs = list(jobs)
    _linalg_ready(mesh.device)
    caller = torch.cuda.current_stream(mesh.device)
    local = threading.local()

    def run(job):
        if not hasattr(local, 'solver'):
            local.solver = FemModeSolver(mesh, **solver_args)
            local.stream = torch.cuda.Stream(mesh.device)
            local.stream.wait_stream(caller)
        n_effs, wl_norm, bloch, shift = job
        with torch.cuda.stream(local.stream):
            out = local.solver.solve_pair(n_effs, wl_norm, bloch, nval, shift=shift, stream=local.stream,
                                          concurrent=False)
            local.stream.synchronize()
        return out

    with cf.ThreadPoolExecutor(max_workers=max(1, int(workers))) as ex:
        results = list(ex.map(run, jobs))
    torch.cuda.synchronize(mesh.device)
    return results
