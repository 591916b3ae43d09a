"""P2 triangular meshes of the unit cell (6-node triangles).

The FEM mode solve and gmsh meshing of the reference stay outside this
package; the overlap kernels only need the element table.  ``Mesh`` holds
the arrays in the reference's conventions (backend/fortran/geometry.f:27-60):
node coordinates in units of the period, ``table_nod`` with 1-based node
numbers (vertices 1-3 then the mid-edge nodes of edges 1-2, 2-3, 3-1) and
1-based material types.  ``Mesh.from_mail`` reads the reference's .mail
files; ``square_cell`` makes a structured mesh with a circular inclusion.
"""
from __future__ import annotations

import numpy as np


class Mesh(object):
    def __init__(self, x, table_nod, type_el, type_nod=None):
        self.x = np.ascontiguousarray(x, np.float64)
        # node types of the .mail file: non-zero on the cell boundary (the FEM
        # solve pairs those nodes periodically)
        self.type_nod = None if type_nod is None else np.ascontiguousarray(type_nod, np.int32)
        self.table_nod = np.ascontiguousarray(table_nod, np.int64)
        self.type_el = np.ascontiguousarray(type_el, np.int64)
        if self.table_nod.ndim != 2 or self.table_nod.shape[1] != 6:
            raise ValueError('table_nod must be [nel][6]')
        if self.table_nod.min() < 1 or self.table_nod.max() > len(self.x):
            raise ValueError('table_nod must hold 1-based node numbers')

    @property
    def npt(self):
        return len(self.x)

    @property
    def nel(self):
        return len(self.table_nod)

    @classmethod
    def from_mail(cls, path):
        """Read a .mail mesh (npt nel; npt rows 'k x y type'; nel rows 'k n1..n6 type')."""
        with open(path) as f:
            tok = f.read().split()
        npt, nel = int(tok[0]), int(tok[1])
        p = 2
        pts = np.array(tok[p:p + 4 * npt], dtype=float).reshape(npt, 4)
        p += 4 * npt
        els = np.array(tok[p:p + 8 * nel], dtype=np.int64).reshape(nel, 8)
        return cls(pts[:, 1:3], els[:, 1:7], els[:, 7], pts[:, 3].astype(np.int32))

    def to_device(self, device='cuda'):
        import torch
        return (torch.tensor(self.x, device=device), torch.tensor(self.table_nod, device=device),
                torch.tensor(self.type_el, device=device))


def square_cell(n, dy=1.0, radius=None, center=(0.5, 0.5), jitter=0.0, seed=0):
    """Structured P2 mesh of [0,1] x [0,dy]: n x n squares, two triangles each
    (2 n^2 elements).  Elements whose centroid lies within ``radius`` of
    ``center`` get type 2, the rest type 1.  ``jitter`` moves interior
    vertices randomly (a fraction of the spacing) to make elements irregular;
    mid-edge nodes stay at edge midpoints (straight-sided elements)."""
    m = n + 1
    xs = np.linspace(0.0, 1.0, m)
    ys = np.linspace(0.0, dy, m)
    X, Y = np.meshgrid(xs, ys, indexing='ij')
    V = np.stack([X.ravel(), Y.ravel()], axis=1)
    if jitter:
        rng = np.random.default_rng(seed)
        inner = (X.ravel() > 0) & (X.ravel() < 1) & (Y.ravel() > 0) & (Y.ravel() < dy)
        V[inner] += jitter * rng.uniform(-0.5, 0.5, (inner.sum(), 2)) * np.array([1.0 / n, dy / n])
    vid = lambda i, j: i * m + j
    tris = []
    for i in range(n):
        for j in range(n):
            a, b, c, d = vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)
            tris.append((a, b, c))
            tris.append((a, c, d))
    tris = np.array(tris, dtype=np.int64)
    edges = {}
    pts = [tuple(v) for v in V]
    coords = list(V)
    table = np.zeros((len(tris), 6), np.int64)
    for e, (a, b, c) in enumerate(tris):
        table[e, :3] = (a, b, c)
        for k, (u, v) in enumerate(((a, b), (b, c), (c, a))):
            key = (min(u, v), max(u, v))
            if key not in edges:
                edges[key] = len(coords)
                coords.append(0.5 * (V[u] + V[v]))
            table[e, 3 + k] = edges[key]
    x = np.array(coords)
    cen = V[tris].mean(axis=1)
    typ = np.ones(len(tris), np.int64)
    if radius is not None:
        r = np.hypot(cen[:, 0] - center[0], cen[:, 1] - center[1])
        typ[r <= radius] = 2
    return Mesh(x, table + 1, typ)


class Mesh1D(object):
    """P2 mesh of a 1D grating's period (backend/fortran/py_calc_modes_1d.f
    conventions): node coordinates ``x`` (the unit the periodic span is
    measured in, the period itself for the drop-in objects), ``table_nod``
    [nel][3] with 1-based node numbers (element ends, then midpoint) and
    1-based material types ``type_el``."""

    def __init__(self, x, table_nod, type_el=None):
        self.x = np.ascontiguousarray(x, np.float64).ravel()
        self.table_nod = np.ascontiguousarray(table_nod, np.int64)
        if self.table_nod.ndim != 2 or self.table_nod.shape[1] != 3:
            raise ValueError('table_nod must be [nel][3]')
        if self.table_nod.min() < 1 or self.table_nod.max() > len(self.x):
            raise ValueError('table_nod must hold 1-based node numbers')
        n = len(self.table_nod)
        self.type_el = np.ones(n, np.int64) if type_el is None else np.ascontiguousarray(type_el, np.int64)

    @property
    def npt(self):
        return len(self.x)

    @property
    def nel(self):
        return len(self.table_nod)

    @property
    def period_x(self):
        """Span of the periodic cell (periodic_cond_1d.f:120-135 takes the
        distance between the two periodic end nodes)."""
        return float(self.x.max() - self.x.min())

    @classmethod
    def uniform(cls, n_el, x0=0.0, x1=1.0, jitter=0.0, seed=0, types=None):
        """n_el elements over [x0, x1] (interior end nodes moved by up to
        ``jitter`` of the spacing); end nodes first, then the midpoints."""
        e = np.linspace(x0, x1, n_el + 1)
        if jitter:
            rng = np.random.default_rng(seed)
            e[1:-1] += jitter * (x1 - x0) / n_el * rng.uniform(-0.5, 0.5, n_el - 1)
        mid = 0.5 * (e[:-1] + e[1:])
        x = np.concatenate([e, mid])
        tab = np.stack([np.arange(1, n_el + 1), np.arange(2, n_el + 2),
                        n_el + 2 + np.arange(n_el)], axis=1)
        return cls(x, tab, types)
