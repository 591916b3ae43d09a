"""ctypes wrapper of oracle/overlap_oracle.c (TEST INFRASTRUCTURE ONLY).

CPU restatement of the reference's overlap integrals (J_overlap.f,
J_dagger_overlap.f), plane-wave ordering (pw_ordering.f) and Bloch-mode
orthogonality / normalisation (orthogonal.f, normalisation.f); see the C
file's header for line citations.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .build import build_oracle

_lib = None
vp = C.c_void_p


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build_oracle())
        _lib.ora_pw_ordering.restype = C.c_int
        _lib.ora_pw_ordering.argtypes = [C.c_int, C.c_double, C.c_double, vp, C.c_double, vp, vp, vp]
        for nm in ('ora_J_overlap', 'ora_J_dagger_overlap'):
            f = getattr(_lib, nm)
            f.restype = None
            f.argtypes = [C.c_long, C.c_long, vp, vp, vp, C.c_double, C.c_double, vp, vp, C.c_int, C.c_int, vp]
        _lib.ora_orthogonal_normalise.restype = C.c_int
        _lib.ora_orthogonal_normalise.argtypes = [C.c_long, C.c_long, vp, vp, vp, vp, vp, vp, vp, vp,
                                                  C.c_double, vp, vp, vp]
    return _lib


def _p(a):
    return a.ctypes.data_as(vp)


def pw_ordering(ordre_ls, d, dy, bloch, k0):
    """(index_pw_inv (0-based), px, py) of the disc orders (pw_ordering.f)."""
    n = (2 * ordre_ls + 1) ** 2
    inv = np.zeros(n, np.int32)
    px = np.zeros(n, np.int32)
    py = np.zeros(n, np.int32)
    b = np.ascontiguousarray(bloch, np.float64)
    m = lib().ora_pw_ordering(int(ordre_ls), float(d), float(dy), _p(b), float(k0), _p(inv), _p(px), _p(py))
    return inv[:m], px[:m], py[:m]


def _sol(sol):
    sol = np.ascontiguousarray(sol, np.complex128)
    if sol.ndim != 4 or sol.shape[2:] != (13, 3):
        raise ValueError('sol must be [nel][nval][13][3]')
    return sol


def J_overlap(x, table_nod, sol, d, dy, bloch, index_pw_inv, ordre_ls):
    sol = _sol(sol)
    nel, nval = sol.shape[:2]
    npw = len(index_pw_inv)
    J = np.zeros((2 * npw, nval), np.complex128)
    x = np.ascontiguousarray(x, np.float64)
    tn = np.ascontiguousarray(table_nod, np.int64)
    inv = np.ascontiguousarray(index_pw_inv, np.int32)
    b = np.ascontiguousarray(bloch, np.float64)
    lib().ora_J_overlap(nval, nel, _p(x), _p(tn), _p(sol), float(d), float(dy), _p(b), _p(inv),
                        int(ordre_ls), npw, _p(J))
    return J


def J_dagger_overlap(x, table_nod, sol, d, dy, bloch, index_pw_inv, ordre_ls):
    sol = _sol(sol)
    nel, nval = sol.shape[:2]
    npw = len(index_pw_inv)
    Jd = np.zeros((nval, 2 * npw), np.complex128)
    x = np.ascontiguousarray(x, np.float64)
    tn = np.ascontiguousarray(table_nod, np.int64)
    inv = np.ascontiguousarray(index_pw_inv, np.int32)
    b = np.ascontiguousarray(bloch, np.float64)
    lib().ora_J_dagger_overlap(nval, nel, _p(x), _p(tn), _p(sol), float(d), float(dy), _p(b), _p(inv),
                               int(ordre_ls), npw, _p(Jd))
    return Jd


def orthogonal_normalise(x, table_nod, type_el, pp, beta1, beta2, sol1, sol2, k0):
    """Returns (ovl, perm, scale, n_warn, sol2_normalised, beta2_reordered)."""
    sol1 = _sol(sol1)
    sol2 = _sol(sol2).copy()
    nel, nval = sol1.shape[:2]
    b1 = np.ascontiguousarray(beta1, np.complex128)
    b2 = np.ascontiguousarray(beta2, np.complex128).copy()
    ovl = np.zeros((nval, nval), np.complex128)
    perm = np.zeros(nval, np.int32)
    scale = np.zeros(nval, np.complex128)
    x = np.ascontiguousarray(x, np.float64)
    tn = np.ascontiguousarray(table_nod, np.int64)
    te = np.ascontiguousarray(type_el, np.int64)
    ppa = np.ascontiguousarray(pp, np.complex128)
    w = lib().ora_orthogonal_normalise(nval, nel, _p(x), _p(tn), _p(te), _p(ppa), _p(b1), _p(b2), _p(sol1),
                                       _p(sol2), float(k0), _p(ovl), _p(perm), _p(scale))
    return ovl, perm, scale, w, sol2, b2
