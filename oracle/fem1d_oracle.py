"""CPU oracle for the FEM Bloch-mode solve of a 1D grating layer.

TEST INFRASTRUCTURE ONLY: a numpy / scipy restatement used as the checker by
``tests/``; the product package ``emustack_b200`` never imports it.

It restates, for the E-field formulation (the reference's only use), the
steps of the reference's calc_modes_1d.  Paths are relative to the EMUstack
source tree:

* pp, qq, the prime (+k) and adjoint (-k) solves  backend/fortran/py_calc_modes_1d.f:330-500
* DOF layout: E_x discontinuous P2 (3 per           backend/fortran/periodic_cond_1d.f:30-160
  element), E_y and E_z continuous P3 (4 per
  element, the end values shared, the last one
  the periodic image of the first)
* element matrices and Bloch phase factors          backend/fortran/asmbly_1d.f:60-300
* element integrals of the P2 / P3 bases            matrix_mxx_1d.f, matrix_kxy_1d.f,
                                                    matrix_kyy_1d.f, matrix_myy_1d.f,
                                                    matrix_kyx_1d.f (here by exact Gauss-Legendre
                                                    quadrature of the Lagrange bases)
* shift-and-invert eigen-solve (ARPACK, 'LM',       backend/fortran/valpr_lapack_1d.f:390-560
  dense LU of K - shift M)
* beta branch, -Re(beta^2) order                    py_calc_modes_1d.f:460-482, z_indexx.f
* nodal values and the normalisation by the         backend/fortran/array_sol_1d.f:60-220
  largest value near the middle of the cell, else
  on its right (prime) or left (adjoint) half

Layout of the result, as the reference's sol(11, nval, nel): per element E_x
at its P2 nodes (x_min, x_max, middle), E_y at its P3 nodes (x_min, x_max,
x_min + h/3, x_min + 2h/3), E_z at the same nodes.

Pinned against the reference's stored results of its test case 4 (two
gratings; tests/golden/case_4.npz) through tests/test_oracle_fem1d.py, with
the mesh and solver inputs the reference passes (tests/golden/fem1d.npz).
"""
from __future__ import annotations

import numpy as np

try:
    from .overlap1d_oracle import z_indexx
except ImportError:  # imported as a top-level module
    from overlap1d_oracle import z_indexx

P2_T = np.array([0.0, 1.0, 0.5])
P3_T = np.array([0.0, 1.0, 1.0 / 3.0, 2.0 / 3.0])


def _lagrange(nodes, t):
    """Values and t-derivatives [len(nodes)][len(t)] of the Lagrange basis."""
    t = np.asarray(t, float)
    n = len(nodes)
    v = np.ones((n, len(t)))
    d = np.zeros((n, len(t)))
    for i in range(n):
        others = [nodes[j] for j in range(n) if j != i]
        den = np.prod([nodes[i] - o for o in others])
        v[i] = np.prod([t - o for o in others], axis=0) / den
        for k, ok in enumerate(others):
            rest = [o for o in others if o is not ok]
            d[i] += np.prod([t - o for o in rest], axis=0) / den if rest else 1.0 / den
    return v, d


def element_integrals():
    """The reference element's integrals on [0, 1] (h = 1): Mxx = int P2 P2,
    Kxy = int P2 (P3)', Kyy = int (P3)' (P3)', Myy = int P3 P3 (an element of
    length h scales Mxx, Myy by h and Kyy by 1/h; Kxy does not scale)."""
    t, w = np.polynomial.legendre.leggauss(6)
    t, w = 0.5 * (t + 1.0), 0.5 * w
    v2, _ = _lagrange(P2_T, t)
    v3, d3 = _lagrange(P3_T, t)
    Mxx = (v2 * w) @ v2.T
    Kxy = (v2 * w) @ d3.T
    Kyy = (d3 * w) @ d3.T
    Myy = (v3 * w) @ v3.T
    return Mxx, Kxy, Kyy, Myy


class Topology1D(object):
    """DOFs of periodic_cond_1d.f: per element 3 E_x values of its own, the
    E_y and E_z values at x_min shared with the element before (the first
    element's with the last element's x_max, a period away); equations
    numbered element by element (E_x, then E_y at x_min, h/3, 2h/3, then E_z
    the same).  ``dof[e][11]`` in the local order of sol; ``shift[e][11]``
    the x offset of a DOF from the one it is an image of (the period for the
    last element's x_max values, else 0)."""

    def __init__(self, x_arr, table_nod):
        tab = np.asarray(table_nod, np.int64)
        if tab.shape[0] == 3 and tab.shape[1] != 3:
            tab = tab.T
        self.table_nod = tab
        self.x = np.asarray(x_arr, float)
        nel = len(tab)
        self.nel = nel
        xmin = self.x[tab[:, 0] - 1]
        xmax = self.x[tab[:, 1] - 1]
        if np.any(xmax <= xmin) or np.any(np.abs(xmin[1:] - xmax[:-1]) > 1e-12 * (xmax[-1] - xmin[0])):
            raise ValueError('the 1D elements must be ordered left to right and contiguous')
        self.xmin, self.xmax = xmin, xmax
        self.period = xmax[-1] - xmin[0]
        dof = np.zeros((nel, 11), np.int64)
        for e in range(nel):
            b = 9 * e
            dof[e, 0:3] = b + np.arange(3)
            dof[e, 3] = b + 3            # E_y at x_min
            dof[e, 5], dof[e, 6] = b + 4, b + 5
            dof[e, 7] = b + 6            # E_z at x_min
            dof[e, 9], dof[e, 10] = b + 7, b + 8
        for e in range(nel):
            nxt = (e + 1) % nel
            dof[e, 4] = dof[nxt, 3]      # E_y at x_max = the next element's x_min
            dof[e, 8] = dof[nxt, 7]
        self.dof = dof
        self.neq = 9 * nel
        self.shift = np.zeros((nel, 11))
        self.shift[nel - 1, 4] = self.shift[nel - 1, 8] = self.period
        h = (xmax - xmin)[:, None]
        self.xloc = np.concatenate([xmin[:, None] + h * P2_T[None], xmin[:, None] + h * P3_T[None],
                                    xmin[:, None] + h * P3_T[None]], axis=1)


def element_matrices(topo, n_eff, type_el, k0, bloch_x, bloch_y):
    """Local K, M [nel][11][11] (trial row, test column) of asmbly_1d.f with
    pp = 1, qq = n^2 k0^2, times val_exp(test) conj(val_exp(trial))."""
    Mxx0, Kxy0, Kyy0, Myy0 = element_integrals()
    Kyx0 = Kxy0.T
    eps = np.asarray(n_eff, complex) ** 2
    qq = eps * k0 ** 2
    pp = np.ones_like(qq)
    nel = topo.nel
    K = np.zeros((nel, 11, 11), complex)
    M = np.zeros((nel, 11, 11), complex)
    X, Y, Z = slice(0, 3), slice(3, 7), slice(7, 11)
    by = bloch_y
    for e in range(nel):
        h = topo.xmax[e] - topo.xmin[e]
        te = int(type_el[e]) - 1
        p, q = pp[te], qq[te]
        Mxx, Kxy, Kyy, Myy, Kyx = Mxx0 * h, Kxy0, Kyy0 / h, Myy0 * h, Kyx0
        K[e, X, X] = (p * by ** 2 - q) * Mxx
        M[e, X, X] = -p * Mxx
        K[e, Y, X] = -1j * by * p * Kyx
        K[e, Z, X] = -p * Kyx
        K[e, X, Y] = 1j * by * p * Kxy
        K[e, Y, Y] = p * Kyy - q * Myy
        M[e, Y, Y] = -p * Myy
        K[e, Z, Y] = 1j * by * p * Myy
        M[e, X, Z] = p * Kxy
        M[e, Y, Z] = 1j * by * p * Myy
        K[e, Z, Z] = p * Kyy + (p * by ** 2 - q) * Myy
    ph = np.exp(1j * bloch_x * topo.shift)
    fac = np.conj(ph)[:, :, None] * ph[:, None, :]
    return K * fac, M * fac


def assemble(topo, K, M):
    import scipy.sparse as sp
    r = np.repeat(topo.dof, 11, axis=1).ravel()
    c = np.tile(topo.dof, (1, 11)).ravel()
    n = topo.neq
    return (sp.csc_matrix((K.ravel(), (r, c)), shape=(n, n)),
            sp.csc_matrix((M.ravel(), (r, c)), shape=(n, n)))


def beta_from(b2):
    b = np.sqrt(np.asarray(b2, complex))
    flip = np.where(np.abs(b.imag) < 1e-8, b.real < 0, b.imag < 0)
    return np.where(flip, -b, b)


def eigen_solve(Kg, Mg, nval, shift):
    import scipy.sparse.linalg as sla
    A = (Kg - shift * Mg).tocsc()
    lu = sla.splu(A)
    op = sla.LinearOperator(A.shape, matvec=lambda v: lu.solve(Mg @ v), dtype=complex)
    nvect = 2 * nval + nval // 2 + 3
    nu, vec = sla.eigs(op, k=nval, which='LM', ncv=min(nvect, A.shape[0] - 1), tol=0,
                       maxiter=max(1000, 30 * nval))
    return 1.0 / nu + shift, vec


def nodal_fields(topo, vec, bloch_x, adjoint):
    """sol [nel][nval][11] from eigenvectors [neq][nval] (array_sol_1d.f):
    each mode divided by its first largest value within a quarter element of
    the cell's middle when that is at least 0.95 of its largest value, else
    by its first largest value right of the middle (prime modes) or left of
    it (adjoint modes)."""
    ph = np.exp(1j * bloch_x * topo.shift)                    # [nel][11]
    sol = vec[topo.dof] * ph[:, :, None]                       # [nel][11][nval]
    sol = sol.transpose(0, 2, 1).copy()                        # [nel][nval][11]
    nel, nval = sol.shape[:2]
    x = topo.xloc
    xlo, xhi = topo.xmin[0], topo.xmax[-1]
    x_mid = 0.5 * (xlo + xhi)
    dx = (xhi - xlo) / nel
    flat = sol.transpose(1, 0, 2).reshape(nval, -1)            # [nval][nel*11], element order
    xf = x.reshape(-1)
    mag = np.abs(flat)

    def first_max(mask):
        m = np.where(mask[None, :], mag, -1.0)
        i = np.argmax(m, axis=1)
        return flat[np.arange(nval), i]

    zmax = first_max(np.ones_like(xf, bool))
    zmid = first_max(np.abs(xf - x_mid) < dx / 4.0)
    zside = first_max(xf < x_mid) if adjoint else first_max(xf > x_mid)
    use_mid = np.abs(zmid / zmax) >= 0.95
    z = np.where(use_mid, zmid, zside)
    return sol / z[None, :, None]


def solve_modes(x_arr, table_nod, type_el, n_eff, wl_norm, bloch_x, bloch_y, nval, shift):
    """beta1, sol1 (+k) and beta2, sol2 (-k) of calc_modes_1d, sorted by
    -Re(beta^2)."""
    topo = Topology1D(x_arr, table_nod)
    k0 = 2 * np.pi / wl_norm
    out = []
    for sgn in (1.0, -1.0):
        K, M = element_matrices(topo, n_eff, type_el, k0, sgn * bloch_x, sgn * bloch_y)
        Kg, Mg = assemble(topo, K, M)
        b2, vec = eigen_solve(Kg, Mg, nval, shift)
        beta = beta_from(b2)
        order = z_indexx(-np.real(beta ** 2))
        beta, vec = beta[order], vec[:, order]
        out += [beta, nodal_fields(topo, vec, sgn * bloch_x, adjoint=sgn < 0)]
    return tuple(out)
