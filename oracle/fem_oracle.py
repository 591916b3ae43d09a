"""CPU oracle for the FEM Bloch-mode solve of a 2D nanostructured layer.

TEST INFRASTRUCTURE ONLY: a numpy / scipy restatement used as the checker by
``tests/``; the product package ``emustack_b200`` never imports it.

It restates, for the E-field formulation with periodic boundary conditions
(the reference's only use), the steps of the reference's calc_modes_2d.
Paths are relative to the EMUstack source tree:

* pp, qq of each material, shift-and-invert   backend/fortran/py_calc_modes.f:243-247, 575-616,
  eigenvalues -> beta (sign rule), sort        :655-690 ; backend/mode_calcs.py:300-310 (shift)
* periodic node pairing (lowest index = origin) backend/fortran/periodic_node.f:60-120
* DOF per entity: face 3, edge 3, P3 node 1    backend/fortran/periodic_cond.f:60-140
* element matrices, Eq. (40) of Dossou &       backend/fortran/asmbly.f:60-330
  Fontaine (CMAME 194, 2005)
* transverse basis (face + 3 edges x 3)        backend/fortran/basis_ls.f, basis_vec.f
* P1 / P2 / P3 Lagrange bases, affine map      phi1_2d_mat.f, phi2_2d_mat.f, phi3_2d_mat.f,
                                               jacobian_p1_2d.f (curved_elem_tri.f:62 makes
                                               every element straight)
* 16-point quadrature                          quad_triangle.f:56-145
* Arnoldi shift-and-invert (ARPACK, 'LM',      backend/fortran/valpr_umf_64.f:300-470
  ncv = 2 nval + nval/2 + 3, tol = 0)
* order of the modes: -Re(beta^2) ascending    z_indexx.f:26-28
* nodal fields, max-modulus normalisation      backend/fortran/array_sol.f:88-300

The global numbering of faces, edges and P3 nodes is this module's own; the
reference's numbering only permutes the unknowns, so eigenvalues and nodal
fields are the same.  Edge orientation follows basis_ls: the end with the
lower (periodically mapped) node number first.

The eigen-solve is scipy's ARPACK (``scipy.sparse.linalg.eigs``) on the
operator (K - shift M)^-1 M with a sparse LU (``splu``), the reference's
shift-and-invert with UMFPACK replaced by SuperLU.

Pinned against the reference's stored results: the Bloch-mode propagation
constants of tests/ref/case_1.npz and case_2.npz (the reference's own mesh
4testing-600_120.mail), and, through the overlap and GSM oracles, their
interface and net reflection matrices (``tests/test_oracle_fem.py``).
"""
from __future__ import annotations

import numpy as np

try:
    from .overlap1d_oracle import z_indexx
except ImportError:  # imported as a top-level module
    from overlap1d_oracle import z_indexx

# 16-point rule on the reference triangle (quad_triangle.f:56-145)
_W = [1.443156076777862e-1 / 2.0] + [2.852749028018549e-1 / 6.0] * 3 + \
     [9.737549286959440e-2 / 6.0] * 3 + [3.096521116041552e-1 / 6.0] * 3 + \
     [1.633818850466092e-1 / 12.0] * 6
_a1, _b1 = 4.592925882927229e-1, 8.141482341455413e-2
_a2, _b2 = 5.054722831703103e-2, 8.989055433659379e-1
_a3, _b3 = 1.705693077517601e-1, 6.588613844964797e-1
_a4, _b4, _c4 = 7.284923929554041e-1, 2.63112829634638689e-1, 8.394777409957211e-3
_c = 1.0 / 3.0
_XQ = [_c, _a1, _a1, _b1, _a2, _a2, _b2, _a3, _a3, _b3, _a4, _b4, _b4, _c4, _c4, _a4]
_YQ = [_c, _a1, _b1, _a1, _a2, _b2, _a2, _a3, _b3, _a3, _b4, _a4, _c4, _b4, _a4, _c4]
QUAD = (np.array(_W), np.array(_XQ), np.array(_YQ))

# the P2 nodes of the reference triangle (interp_nod_2d.f)
P2_NODES = np.array([[0, 0], [1, 0], [0, 1], [0.5, 0], [0.5, 0.5], [0, 0.5]], dtype=float)
# local edges (end nodes, 0-based) in basis_ls order: (1,2), (2,3), (1,3); mid nodes 4, 5, 6
EDGES = ((0, 1), (1, 2), (0, 2))
# P3 edge nodes: (local edge, local vertex it lies next to), phi3_2d_mat.f nodes 4-9
P3_EDGE_NODES = ((0, 0), (0, 1), (1, 1), (1, 2), (2, 2), (2, 0))


def read_mail(path):
    """x [npt][2], node type [npt] (non-zero on the cell boundary), table_nod
    [nel][6] (1-based), type_el [nel] of a .mail mesh."""
    with open(path) as f:
        tok = f.read().split()
    npt, nel = int(tok[0]), int(tok[1])
    p = 2
    pts = np.array(tok[p:p + 4 * npt], dtype=float).reshape(npt, 4)
    p += 4 * npt
    els = np.array(tok[p:p + 8 * nel], dtype=np.int64).reshape(nel, 8)
    return pts[:, 1:3].copy(), pts[:, 3].astype(np.int64), els[:, 1:7].copy(), els[:, 7].copy()


def phi1(x, y):
    """P1 values and gradients (phi1_2d_mat.f)."""
    v = np.array([1 - x - y, x, y])
    g = np.array([[-1.0, 1.0, 0.0], [-1.0, 0.0, 1.0]])
    return v, g


def phi2(x, y):
    """P2 values [6] and gradients [2][6] (phi2_2d_mat.f)."""
    v = np.array([(-1 + x + y) * (-1 + 2 * x + 2 * y), x * (-1 + 2 * x), y * (-1 + 2 * y),
                  -4 * x * (-1 + x + y), 4 * x * y, -4 * y * (-1 + x + y)])
    g = np.array([[-3 + 4 * x + 4 * y, -1 + 4 * x, 0, 4 - 8 * x - 4 * y, 4 * y, -4 * y],
                  [-3 + 4 * x + 4 * y, 0, -1 + 4 * y, -4 * x, 4 * x, 4 - 4 * x - 8 * y]], dtype=float)
    return v, g


def phi3(x, y):
    """P3 values [10] and gradients [2][10] (phi3_2d_mat.f)."""
    v = np.array([
        -((-1 + x + y) * (-2 + 3 * x + 3 * y) * (-1 + 3 * x + 3 * y)) / 2.,
        (x * (-2 + 3 * x) * (-1 + 3 * x)) / 2.,
        (y * (-2 + 3 * y) * (-1 + 3 * y)) / 2.,
        (9 * x * (-1 + x + y) * (-2 + 3 * x + 3 * y)) / 2.,
        (-9 * x * (-1 + 3 * x) * (-1 + x + y)) / 2.,
        (9 * x * (-1 + 3 * x) * y) / 2.,
        (9 * x * y * (-1 + 3 * y)) / 2.,
        (-9 * y * (-1 + x + y) * (-1 + 3 * y)) / 2.,
        (9 * y * (-1 + x + y) * (-2 + 3 * x + 3 * y)) / 2.,
        -27 * x * y * (-1 + x + y)])
    t = (-11 - 27 * x * x + x * (36 - 54 * y) + 36 * y - 27 * y * y) / 2.
    g = np.array([
        [t, 1 - 9 * x + (27 * x * x) / 2., 0,
         (9 * (2 + 9 * x * x - 5 * y + 3 * y * y + 2 * x * (-5 + 6 * y))) / 2.,
         (-9 * (1 + 9 * x * x - y + x * (-8 + 6 * y))) / 2.,
         (9 * (-1 + 6 * x) * y) / 2., (9 * y * (-1 + 3 * y)) / 2., (-9 * y * (-1 + 3 * y)) / 2.,
         (9 * y * (-5 + 6 * x + 6 * y)) / 2., -27 * y * (-1 + 2 * x + y)],
        [t, 0, 1 - 9 * y + (27 * y * y) / 2.,
         (9 * x * (-5 + 6 * x + 6 * y)) / 2., (-9 * x * (-1 + 3 * x)) / 2., (9 * x * (-1 + 3 * x)) / 2.,
         (9 * x * (-1 + 6 * y)) / 2., (-9 * (1 - 8 * y + 9 * y * y + x * (-1 + 6 * y))) / 2.,
         (9 * (2 + 3 * x * x - 10 * y + 9 * y * y + x * (-5 + 12 * y))) / 2.,
         -27 * x * (-1 + x + 2 * y)]])
    return v, g


def periodic_nodes(x, type_nod, tol=1e-6):
    """Origin node (0-based, itself for a non-periodic node) and the lattice
    shift x[i] - x[origin] of every node, paired as periodic_node.f pairs
    them: boundary nodes in index order, the first of a class its origin,
    two nodes paired when their difference is a lattice vector ix a1 + iy a2
    (ix, iy in -1..1) within tol in the 1-norm."""
    npt = len(x)
    xmin, xmax = x[:, 0].min(), x[:, 0].max()
    ymin, ymax = x[:, 1].min(), x[:, 1].max()
    a1 = np.array([xmax - xmin, 0.0])
    a2 = np.array([0.0, ymax - ymin])
    vecs = [ix * a1 + iy * a2 for ix in (-1, 0, 1) for iy in (-1, 0, 1)]
    ip = np.full(npt, -1, np.int64)
    bnd = np.nonzero(type_nod != 0)[0]
    for ii, i in enumerate(bnd[:-1]):
        for j in bnd[ii + 1:]:
            if ip[j] != -1:
                continue
            d = x[j] - x[i]
            if any(np.abs(d - v).sum() < tol for v in vecs):
                if ip[i] == -1:
                    ip[i] = i
                    ip[j] = i
                else:
                    ip[j] = ip[i]
    if np.any(ip[bnd] == -1):
        raise ValueError('a boundary node has no periodic image')
    origin = np.where(ip >= 0, ip, np.arange(npt))
    return origin, x - x[origin], (a1, a2)


class Topology(object):
    """DOF numbering of the mixed element (asmbly.f: 14 entities per element,
    face and 3 edges with 3 transverse DOFs each, 10 P3 nodes with one E_z
    DOF): ``dof[e][22]`` (12 transverse then 10 z, 0-based), the lattice
    shift of each of the 14 entity instances ``shift[e][14][2]`` (its
    position minus its origin's, the argument of the Bloch phase), and the
    edge ends in basis_ls order ``ends[e][3][2]`` (local vertices, lower
    mapped node number first)."""

    def __init__(self, x, type_nod, table_nod):
        nel = len(table_nod)
        t = np.asarray(table_nod, np.int64) - 1
        origin, shift, self.lattice = periodic_nodes(x, type_nod)
        tm = origin[t]                       # periodically mapped node numbers
        keys = {}

        def num(key, width):
            if key not in keys:
                keys[key] = (len(keys), width)
            return keys[key][0]

        ent = np.zeros((nel, 14), np.int64)
        self.shift = np.zeros((nel, 14, 2))
        self.ends = np.zeros((nel, 3, 2), np.int64)
        for e in range(nel):
            ent[e, 0] = num(('f', e), 3)
            for k, (p, q) in enumerate(EDGES):
                mid = t[e, 3 + k]
                ent[e, 1 + k] = num(('e', origin[mid]), 3)
                self.shift[e, 1 + k] = shift[mid]
                self.ends[e, k] = (p, q) if tm[e, p] <= tm[e, q] else (q, p)
                if tm[e, p] == tm[e, q]:
                    raise ValueError('an edge whose ends are periodic images of each other')
            for v in range(3):
                ent[e, 4 + v] = num(('v', tm[e, v]), 1)
                self.shift[e, 4 + v] = shift[t[e, v]]
            for n, (k, v) in enumerate(P3_EDGE_NODES):
                mid = t[e, 3 + k]
                ent[e, 7 + n] = num(('p', origin[mid], tm[e, v]), 1)
                self.shift[e, 7 + n] = shift[mid]
            ent[e, 13] = num(('i', e), 1)
        # equation numbers: 3 per face / edge class, 1 per P3 node class
        first = np.zeros(len(keys), np.int64)
        width = np.zeros(len(keys), np.int64)
        for key, (idx, w) in keys.items():
            width[idx] = w
        first[1:] = np.cumsum(width)[:-1]
        self.neq = int(width.sum())
        dof = np.zeros((nel, 22), np.int64)
        for k in range(4):
            for q in range(3):
                dof[:, 3 * k + q] = first[ent[:, k]] + q
        dof[:, 12:] = first[ent[:, 4:]]
        self.dof = dof
        self.entity = ent
        self.x, self.table_nod, self.nel = x, np.asarray(table_nod, np.int64), nel


def _element_geometry(x, table_nod):
    """Affine map of each element from its vertices (jacobian_p1_2d.f):
    det [nel], T = B^-1 [nel][2][2]."""
    t = table_nod - 1
    x1, x2, x3 = x[t[:, 0]], x[t[:, 1]], x[t[:, 2]]
    B = np.stack([np.stack([x2[:, 0] - x1[:, 0], x3[:, 0] - x1[:, 0]], 1),
                  np.stack([x2[:, 1] - x1[:, 1], x3[:, 1] - x1[:, 1]], 1)], 1)
    det = B[:, 0, 0] * B[:, 1, 1] - B[:, 0, 1] * B[:, 1, 0]
    T = np.stack([np.stack([B[:, 1, 1], -B[:, 0, 1]], 1),
                  np.stack([-B[:, 1, 0], B[:, 0, 0]], 1)], 1) / det[:, None, None]
    return det, T


def transverse_basis(ends, g1, v2, g2):
    """The 12 transverse basis vectors [12][2] and their curls [12] of one
    element at one point (basis_ls.f, basis_vec.f): face functions
    phi2(mid j) grad(lambda opposite), then per edge (j1, j2) phi2(j1)
    grad(lambda j2), phi2(j2) grad(lambda j1), phi2(mid)(grad lambda j1 -
    grad lambda j2).  g1, g2: P1 / P2 gradients on the element [2][3],
    [2][6]; v2: P2 values."""
    vec = np.zeros((12, 2))
    curl = np.zeros(12)

    def put(i, m, gp1):
        vec[i] = v2[m] * gp1
        curl[i] = g2[0, m] * gp1[1] - g2[1, m] * gp1[0]

    for j in range(3):
        put(j, 3 + j, g1[:, (j + 2) % 3])
    for k in range(3):
        j1, j2 = ends[k]
        put(3 + 3 * k, j1, g1[:, j2])
        put(4 + 3 * k, j2, g1[:, j1])
        put(5 + 3 * k, 3 + k, g1[:, j1] - g1[:, j2])
    return vec, curl


def element_matrices(topo, x, n_eff, type_el, k0, bloch):
    """Local K and M [nel][22][22] (trial row, test column), pp = 1 and
    qq = n^2 k0^2 (E-field formulation), times the Bloch phase factor
    val_exp(test) conj(val_exp(trial)) (asmbly.f:130-320)."""
    det, T = _element_geometry(x, topo.table_nod)
    nel = topo.nel
    eps = np.asarray(n_eff, complex) ** 2
    qq = eps * k0 ** 2
    pp = np.ones_like(qq)
    W, XQ, YQ = QUAD
    K = np.zeros((nel, 22, 22), complex)
    M = np.zeros((nel, 22, 22), complex)
    val_exp = np.exp(1j * (topo.shift @ np.asarray(bloch, float)))   # [nel][14]
    ent_of = np.array([0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 3] + list(range(4, 14)))
    for e in range(nel):
        te = type_el[e] - 1
        vt = np.zeros((12, 2))
        for q in range(16):
            v1, g10 = phi1(XQ[q], YQ[q])
            v2, g20 = phi2(XQ[q], YQ[q])
            v3, g30 = phi3(XQ[q], YQ[q])
            Tt = T[e].T
            g1, g2, g3 = Tt @ g10, Tt @ g20, Tt @ g30
            vt, ct = transverse_basis(topo.ends[e], g1, v2, g2)
            w = W[q] * abs(det[e])
            dtt = vt @ vt.T
            Kq = np.zeros((22, 22), complex)
            Mq = np.zeros((22, 22), complex)
            Kq[:12, :12] = np.outer(ct, ct) * pp[te] - dtt * qq[te]
            Mq[:12, :12] = -dtt * pp[te]
            Mq[:12, 12:] = (vt @ g3) * pp[te]             # trial transverse, test z
            Kq[12:, :12] = (g3.T @ vt.T) * pp[te]         # trial z, test transverse
            Kq[12:, 12:] = -(g3.T @ g3) * pp[te] + np.outer(v3, v3) * qq[te]
            K[e] += Kq * w
            M[e] += Mq * w
        ph = val_exp[e, ent_of]
        fac = np.conj(ph)[:, None] * ph[None, :]
        K[e] *= fac
        M[e] *= fac
    return K, M


def assemble(topo, K, M):
    """Global sparse K and M (rows = trial DOF, columns = test DOF)."""
    import scipy.sparse as sp
    r = np.repeat(topo.dof, 22, axis=1).ravel()
    c = np.tile(topo.dof, (1, 22)).ravel()
    n = topo.neq
    return (sp.csc_matrix((K.ravel(), (r, c)), shape=(n, n)),
            sp.csc_matrix((M.ravel(), (r, c)), shape=(n, n)))


def shift_of(n_eff, k0, bloch):
    """Shift of the shift-and-invert solve (backend/mode_calcs.py:300-310)."""
    return 1.1 * np.real(np.asarray(n_eff)).max() ** 2 * k0 ** 2 - bloch[0] ** 2 - bloch[1] ** 2


def eigen_solve(Kg, Mg, nval, shift, v0=None):
    """The nval eigenvalues of (K - shift M)^-1 M of largest modulus and
    their eigenvectors; returns beta^2 = 1/nu + shift [nval], vectors
    [neq][nval]."""
    import scipy.sparse.linalg as sla
    A = (Kg - shift * Mg).tocsc()
    lu = sla.splu(A)
    op = sla.LinearOperator(A.shape, matvec=lambda v: lu.solve(Mg @ v), dtype=complex)
    nvect = 2 * nval + nval // 2 + 3
    nu, vec = sla.eigs(op, k=nval, which='LM', ncv=min(nvect, A.shape[0] - 1), tol=0, v0=v0,
                       maxiter=max(1000, 30 * nval))
    return 1.0 / nu + shift, vec


def beta_from(b2):
    """beta = sqrt(beta^2) with the reference's branch (py_calc_modes.f:664-674)."""
    b = np.sqrt(np.asarray(b2, complex))
    flip = np.where(np.abs(b.imag) < 1e-8, b.real < 0, b.imag < 0)
    return np.where(flip, -b, b)


def nodal_fields(topo, vec, bloch):
    """sol [nel][nval][13][3] from eigenvectors [neq][nval] (array_sol.f):
    E_x, E_y, E_z at the six P2 nodes (E_z interpolated from the P3 values),
    then E_z at P3 nodes 4-10; every mode divided by its first
    largest-modulus P2-node component."""
    det, T = _element_geometry(topo.x, topo.table_nod)
    nel, nval = topo.nel, vec.shape[1]
    val_exp = np.exp(1j * (topo.shift @ np.asarray(bloch, float)))
    ent_of = np.array([0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 3] + list(range(4, 14)))
    sol = np.zeros((nel, nval, 13, 3), complex)
    # which P2 node each transverse function lives on (basis_list(2, ., .))
    for e in range(nel):
        u = vec[topo.dof[e]] * val_exp[e, ent_of][:, None]      # [22][nval]
        ends = topo.ends[e]
        node_of = [3, 4, 5]
        for k in range(3):
            node_of += [ends[k][0], ends[k][1], 3 + k]
        for inod in range(6):
            xx, yy = P2_NODES[inod]
            v1, g10 = phi1(xx, yy)
            v2, g20 = phi2(xx, yy)
            v3, _ = phi3(xx, yy)
            Tt = T[e].T
            vt, _ = transverse_basis(ends, Tt @ g10, v2, Tt @ g20)
            for i in range(12):
                if node_of[i] == inod:
                    sol[e, :, inod, 0] += u[i] * vt[i, 0]
                    sol[e, :, inod, 1] += u[i] * vt[i, 1]
            for i in range(10):
                sol[e, :, inod, 2] += u[12 + i] * v3[i]
        sol[e, :, 6:13, 2] = u[15:22].T
    # first largest modulus over elements, P2 nodes, components (strict <)
    flat = sol[:, :, :6, :].transpose(1, 0, 2, 3).reshape(nval, -1)
    idx = np.argmax(np.abs(flat), axis=1)
    zmax = flat[np.arange(nval), idx]
    return sol / zmax[None, :, None, None]


def solve_modes(x, type_nod, table_nod, type_el, n_eff, wl_norm, bloch, nval, shift=None,
                topo=None):
    """Bloch modes of one layer for the Bloch vector ``bloch`` and its
    adjoint (-bloch), as calc_modes_2d computes them: returns beta1, sol1,
    beta2, sol2 (modes sorted by -Re(beta^2))."""
    topo = topo or Topology(x, type_nod, table_nod)
    k0 = 2 * np.pi / wl_norm
    if shift is None:
        shift = shift_of(n_eff, k0, bloch)
    out = []
    for sgn in (1.0, -1.0):
        bk = sgn * np.asarray(bloch, float)
        K, M = element_matrices(topo, x, n_eff, type_el, k0, bk)
        Kg, Mg = assemble(topo, K, M)
        b2, vec = eigen_solve(Kg, Mg, nval, shift)
        beta = beta_from(b2)
        order = z_indexx(-np.real(beta ** 2))
        beta, vec = beta[order], vec[:, order]
        out += [beta, nodal_fields(topo, vec, bk)]
    return tuple(out)
