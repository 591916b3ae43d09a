"""Dense GSM path on the GPU: interfaces of nanostructured layers, the
cascade and the energy fluxes (backend/mode_calcs.py:416-515,
backend/stack.py:162-426), batched over spectral points.

``interface_dense`` and ``film_interface`` compute air/layer scattering
matrices; ``DenseStackSolver`` runs the cascade + fluxes of a batch of
stacks that share layer shapes; ``calc_scat_dense`` drives one reference
``Stack`` through them.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import EmuC128, EmuLayer, EmuStackDense, check, lib, ptr, stream_ptr

c128 = torch.complex128


def _dev():
    return torch.device('cuda', torch.cuda.current_device())


def _c(x):
    return EmuC128(float(np.real(x)), float(np.imag(x)))


def _need(t, dtype, name, ndim=None):
    """Fail loudly on tensors the C ABI would misread."""
    if t is None or not t.is_cuda or t.dtype != dtype or not t.is_contiguous():
        raise TypeError('%s must be a contiguous CUDA %s tensor' % (name, dtype))
    if ndim is not None and t.dim() != ndim:
        raise ValueError('%s must have %d dimensions' % (name, ndim))


def zgemm_batched(A, B, C_=None, alpha=1.0, beta=0.0):
    """C = alpha A B + beta C for batched row-major complex128 tensors [b, m, k] x [b, k, n]."""
    _need(A, c128, 'A', 3)
    _need(B, c128, 'B', 3)
    bsz, m, k = A.shape
    n = B.shape[2]
    if B.shape[:2] != (bsz, k):
        raise ValueError('inner dimensions differ')
    if C_ is None:
        C_ = torch.zeros((bsz, m, n), dtype=c128, device=A.device)
    check(lib().emu_zgemm_batched(m, n, k, _c(alpha), ptr(A), k, m * k, ptr(B), n, k * n, _c(beta),
                                  ptr(C_), n, m * n, bsz, stream_ptr()), 'emu_zgemm_batched')
    return C_


def zgesv_batched(A, B):
    """Solve A X = B in place (A overwritten with its LU); returns (X, ipiv, info)."""
    _need(A, c128, 'A', 3)
    _need(B, c128, 'B', 3)
    bsz, n, _ = A.shape
    nrhs = B.shape[2]
    ipiv = torch.empty((bsz, n), dtype=torch.int32, device=A.device)
    info = torch.empty((bsz,), dtype=torch.int32, device=A.device)
    check(lib().emu_zgesv_batched(n, nrhs, ptr(A), n, n * n, ptr(ipiv), ptr(B), nrhs, n * nrhs,
                                  ptr(info), bsz, stream_ptr()), 'emu_zgesv_batched')
    return B, ipiv, info


def film_interface(kz1, n1, kz2, n2, wl_norm):
    """Diagonal film/film interface (backend/mode_calcs.py:451-477).

    kz1, kz2: complex128 [B, Npw] sorted k_z of both films (1 = the incidence
    side, the air reference in a Stack); n1, n2: complex128 [B]; wl_norm
    float64 [B].  Returns R12, T12 diagonals [B, 2 Npw] (R21 = -R12, T21 = T12).
    """
    for t, nm in ((kz1, 'kz1'), (n1, 'n1'), (kz2, 'kz2'), (n2, 'n2')):
        _need(t, c128, nm)
    _need(wl_norm, torch.float64, 'wl_norm')
    B, npw = kz1.shape
    R12 = torch.empty((B, 2 * npw), dtype=c128, device=kz1.device)
    T12 = torch.empty_like(R12)
    check(lib().emu_film_interface_batch(B, npw, ptr(kz1), ptr(n1), ptr(kz2), ptr(n2), ptr(wl_norm),
                                         ptr(R12), ptr(T12), stream_ptr()), 'emu_film_interface_batch')
    return R12, T12


def interface_dense(film_kz, film_n, wl_norm, J, J_dag):
    """Film/nanostructure interface (backend/mode_calcs.py:480-515), batched.

    film_kz complex128 [B, P/2]; film_n complex128 [B]; wl_norm float64 [B];
    J complex128 [B, P, M] (divided by the area ratio); J_dag [B, M, P].
    Returns R12 [B,P,P], T12 [B,M,P], R21 [B,M,M], T21 [B,P,M] and info [B].
    """
    for t, nm in ((film_kz, 'film_kz'), (film_n, 'film_n'), (J, 'J'), (J_dag, 'J_dag')):
        _need(t, c128, nm)
    _need(wl_norm, torch.float64, 'wl_norm')
    B, P, M = J.shape
    if tuple(J_dag.shape) != (B, M, P) or tuple(film_kz.shape) != (B, P // 2):
        raise ValueError('inconsistent interface shapes')
    dev = J.device
    R12 = torch.empty((B, P, P), dtype=c128, device=dev)
    T12 = torch.empty((B, M, P), dtype=c128, device=dev)
    R21 = torch.empty((B, M, M), dtype=c128, device=dev)
    T21 = torch.empty((B, P, M), dtype=c128, device=dev)
    info = torch.empty((B,), dtype=torch.int32, device=dev)
    L = lib()
    nbytes = L.emu_interface_dense_workspace_size(B, P, M)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    check(L.emu_interface_dense_batch(B, P, M, ptr(film_kz), ptr(film_n), ptr(wl_norm), ptr(J),
                                      ptr(J_dag), ptr(R12), ptr(T12), ptr(R21), ptr(T21), ptr(info),
                                      ptr(ws), C.c_size_t(nbytes), stream_ptr()),
          'emu_interface_dense_batch')
    return R12, T12, R21, T21, info


class DenseLayer(object):
    """One layer of a dense batch: device interface matrices with air.

    dense=False: film, R12..T21 are diagonals [B, P]; dense=True: full
    matrices [B, P, P], [B, M, P], [B, M, M], [B, P, M] (a leading 1 instead
    of B shares one matrix across the batch).  kz [B, M] and height_norm
    (height / period) for finite layers: one float for the whole batch, or a
    CUDA float64 tensor [B] of per-point heights.
    """

    def __init__(self, R12, T12, R21, T21, dense, kz=None, height_norm=0.0):
        self.R12, self.T12, self.R21, self.T21 = R12, T12, R21, T21
        self.dense = bool(dense)
        self.kz = kz
        if torch.is_tensor(height_norm):
            _need(height_norm, torch.float64, 'height_norm', 1)
            self.height_norm = height_norm
        else:
            self.height_norm = float(height_norm)
        self.M = int(T12.shape[1]) if dense else int(R12.shape[1])


class DenseStackSolver(object):
    """Cascade + fluxes for a batch of stacks with identical layer shapes."""

    def __init__(self, device=None):
        self.device = device or _dev()
        self._ws = None

    def solve(self, layers, P, pol='TE', incoming=None, specular=None, num_prop=None,
              calc_fluxes=True, shears=None, air_alphas=None, air_betas=None,
              want_vec_coef=False, save_lists=False, mode=0):
        """mode: 0 automatic, 1 one CTA per solve, 2 every step spread over
        many CTAs (emu_stack_dense_batch); results are identical."""
        L = len(layers)
        B = int(layers[0].R12.shape[0])
        dev = self.device
        arr = (EmuLayer * L)()
        for i, ly in enumerate(layers):
            for nm in ('R12', 'T12', 'R21', 'T21'):
                _need(getattr(ly, nm), c128, 'layer %d %s' % (i, nm))
            if ly.kz is not None:
                _need(ly.kz, c128, 'layer %d kz' % i)
            e = arr[i]
            e.M = ly.M
            e.dense = int(ly.dense)
            for nm in ('R12', 'T12', 'R21', 'T21'):
                t = getattr(ly, nm)
                setattr(e, 'd_' + nm, ptr(t))
                setattr(e, 'stride_' + nm, int(t[0].numel()) if t.shape[0] == B and B > 1 else 0)
            if ly.kz is not None:
                e.d_kz = ptr(ly.kz)
                e.stride_kz = int(ly.kz[0].numel()) if ly.kz.shape[0] == B and B > 1 else 0
            if torch.is_tensor(ly.height_norm):
                if ly.height_norm.numel() != B:
                    raise ValueError('layer %d: height_norm must have one entry per point' % i)
                e.d_height_norm = ptr(ly.height_norm)
            else:
                e.height_norm = ly.height_norm
        d = EmuStackDense()
        d.batch, d.n_layers, d.P = B, L, P
        d.mode = int(mode)
        d.h_layers = C.cast(arr, C.POINTER(EmuLayer))
        sh_arr = None
        if shears is not None:
            sh = np.zeros((L, 2), dtype=np.float64)
            for i, s in enumerate(shears):
                s = np.asarray(s, dtype=np.float64).ravel()
                sh[i, :len(s)] = s
            sh_arr = (C.c_double * (2 * L))(*sh.ravel())
            d.h_shears = C.cast(sh_arr, C.POINTER(C.c_double))
            d.shear_ncoord = len(np.asarray(shears[0]).ravel())
            d.d_air_alphas = ptr(air_alphas)
            d.d_air_betas = ptr(air_betas) if air_betas is not None else None
        M0 = layers[0].M
        out = {
            'R_net': torch.empty((B, P, P), dtype=c128, device=dev),
            'T_net': torch.empty((B, M0, P), dtype=c128, device=dev),
            'info': torch.empty((B,), dtype=torch.int32, device=dev),
        }
        d.d_R_net, d.d_T_net, d.d_info = ptr(out['R_net']), ptr(out['T_net']), ptr(out['info'])
        d.calc_fluxes = int(calc_fluxes)
        if calc_fluxes:
            out['fluxes'] = torch.empty((B, L + 1, 2), dtype=torch.float64, device=dev)
            out['flags'] = torch.empty((B,), dtype=torch.int32, device=dev)
            d.d_fluxes, d.d_flags = ptr(out['fluxes']), ptr(out['flags'])
            if not layers[0].dense:
                out['a_list'] = torch.empty((B, L - 1), dtype=torch.float64, device=dev)
                out['t_list'] = torch.empty((B, L - 1), dtype=torch.float64, device=dev)
                out['r_list'] = torch.empty((B,), dtype=torch.float64, device=dev)
                d.d_a_list, d.d_t_list, d.d_r_list = ptr(out['a_list']), ptr(out['t_list']), ptr(out['r_list'])
            if incoming is not None:
                d.pol = _lib.POL_INCOMING
                d.d_incoming = ptr(incoming)
            else:
                d.pol = _lib.POL[pol]
            d.d_specular = ptr(specular)
            d.d_num_prop = ptr(num_prop)
            if want_vec_coef:
                Ms = [layers[k].M for k in range(L - 2, 0, -1)]
                nd = P + sum(Ms) + M0
                nu = P + sum(Ms)
                out['vec_coef_down'] = torch.zeros((B, nd), dtype=c128, device=dev)
                out['vec_coef_up'] = torch.zeros((B, nu), dtype=c128, device=dev)
                d.d_vec_coef_down, d.d_vec_coef_up = ptr(out['vec_coef_down']), ptr(out['vec_coef_up'])
                d.vec_coef_down_stride, d.vec_coef_up_stride = nd, nu
                out['vec_coef_lens'] = ([P] + Ms + [M0], [P] + Ms)
        L_ = lib()
        if save_lists:
            stride = L_.emu_stack_dense_list_stride(C.byref(d))
            out['tnet_list'] = torch.zeros((B, 2 * L - 2, stride), dtype=c128, device=dev)
            out['rnet_list'] = torch.zeros((B, 2 * L - 2, stride), dtype=c128, device=dev)
            d.save_lists = 1
            d.d_tnet_list, d.d_rnet_list = ptr(out['tnet_list']), ptr(out['rnet_list'])
        nbytes = L_.emu_stack_dense_workspace_size(C.byref(d))
        if nbytes == 0:
            raise _lib.EmuError(_lib.EMU_OK + 2, 'emu_stack_dense_workspace_size')
        if self._ws is None or self._ws.numel() < nbytes:
            self._ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        check(L_.emu_stack_dense_batch(C.byref(d), ptr(self._ws), C.c_size_t(self._ws.numel()),
                                       stream_ptr()), 'emu_stack_dense_batch')
        return out


# ---------------------------------------------------------------------------
# drop-in driver for one reference Stack
# ---------------------------------------------------------------------------

def layer_interface(air, lay):
    """Device (R12, T12, R21, T21, dense) of lay with the air reference,
    memoised like backend/mode_calcs.py:416-448 (keyed by object ids)."""
    from .mode_calcs import _interfaces_i_have_known, film_n, is_film
    key = (id(air), id(lay))
    hit = _interfaces_i_have_known.get(key)
    if hit is not None and 'dev' in hit:
        return hit['dev']
    dev = _dev()
    npw = len(air.k_z) // 2
    wln = torch.tensor([air.wl_norm()], dtype=torch.float64, device=dev)
    air_kz = torch.tensor(np.asarray(air.k_z[:npw]).reshape(1, npw), dtype=c128, device=dev)
    air_n = torch.tensor([complex(np.asarray(air.n()).item())], dtype=c128, device=dev)
    if is_film(lay):
        if len(lay.k_z) != len(air.k_z):
            raise ValueError('Need the same number of plane waves in Anallos')
        kz2 = torch.tensor(np.asarray(lay.k_z[:npw]).reshape(1, npw), dtype=c128, device=dev)
        n2 = torch.tensor([film_n(lay)], dtype=c128, device=dev)
        R12, T12 = film_interface(air_kz, air_n, kz2, n2, wln)
        res = (R12, T12, -R12, T12, False)
    else:
        J = torch.tensor(np.ascontiguousarray(lay.J), dtype=c128, device=dev).unsqueeze(0)
        Jd = torch.tensor(np.ascontiguousarray(lay.J_dag), dtype=c128, device=dev).unsqueeze(0)
        if J.shape[1] != 2 * npw:
            raise ValueError("Scattering matrices of layers are not consistent,"
                             "\nsome layers are 1D and others 2D. Check that world_1d status.")
        R12, T12, R21, T21, info = interface_dense(air_kz, air_n, wln, J, Jd)
        if int(info.item()) != 0:
            raise np.linalg.LinAlgError('Singular matrix')
        res = (R12, T12, R21, T21, True)
    _interfaces_i_have_known[key] = {'dev': res}
    return res


def _host_matrices(res):
    R12, T12, R21, T21, dense = res
    if dense:
        return tuple(np.asmatrix(t[0].cpu().numpy()) for t in (R12, T12, R21, T21))
    return tuple(np.asmatrix(np.diag(t[0].cpu().numpy())) for t in (R12, T12, R21, T21))


def calc_scat_dense(stack, pol='TE', incoming_amplitudes=None, calc_fluxes=True,
                    save_scat_list=False):
    """Stack.calc_scat for stacks with nanostructured layers (or when the
    intermediate lists are requested), on the GPU."""
    from .mode_calcs import is_film
    layers = stack.layers
    L = len(layers)
    air = layers[-1].air_ref()
    P = len(air.k_z)
    dev = _dev()
    dl = []
    hs = stack.heights_nm()
    for i, lay in enumerate(layers):
        res = layer_interface(air, lay)
        lay.R12, lay.T12, lay.R21, lay.T21 = _host_matrices(res)
        R12, T12, R21, T21, dense = res
        kz = None
        hn = 0.0
        if 0 < i < L - 1:
            kz = torch.tensor(np.asarray(lay.k_z).reshape(1, -1), dtype=c128, device=dev)
            hn = hs[i - 1] / stack.period
        dl.append(DenseLayer(R12, T12, R21, T21, dense, kz, hn))
    top = layers[-1]
    if calc_fluxes and not is_film(top):
        raise NotImplementedError('energy fluxes need a ThinFilm superstrate')
    spec = torch.tensor([int(getattr(top, 'specular_order', 0))], dtype=torch.int32, device=dev)
    sub = layers[0]
    nprop = torch.tensor([[air.num_prop_pw_per_pol, getattr(top, 'num_prop_pw_per_pol', 0),
                           sub.num_prop_pw_per_pol if is_film(sub) else 0]],
                         dtype=torch.int32, device=dev)
    inc = None
    if incoming_amplitudes is not None:
        inc = torch.tensor(np.asarray(incoming_amplitudes, dtype=np.complex128).reshape(1, -1), device=dev)
    alphas = betas = None
    if stack.shears is not None:
        alphas = torch.tensor(np.asarray(air.alphas, dtype=np.float64).reshape(1, -1), device=dev)
        if not stack.layers[0].structure.world_1d:
            betas = torch.tensor(np.asarray(air.betas, dtype=np.float64).reshape(1, -1), device=dev)
    out = DenseStackSolver(dev).solve(dl, P, pol=pol, incoming=inc, specular=spec, num_prop=nprop,
                                      calc_fluxes=calc_fluxes, shears=stack.shears,
                                      air_alphas=alphas, air_betas=betas,
                                      want_vec_coef=calc_fluxes, save_lists=save_scat_list)
    info = int(out['info'][0].item())
    if info != 0:
        raise np.linalg.LinAlgError('Singular matrix')
    M0 = dl[0].M
    stack.R_net = np.asmatrix(out['R_net'][0].cpu().numpy())
    stack.T_net = np.asmatrix(out['T_net'][0].cpu().numpy())
    if save_scat_list:
        tl = out['tnet_list'][0].cpu().numpy()
        rl = out['rnet_list'][0].cpu().numpy()
        shapes_r, shapes_t = [(P, P)], [(M0, P)]
        for i in range(1, L):
            M = dl[i].M
            shapes_r.append((M, M))
            shapes_t.append((M0, M))
            if i == L - 1:
                break
            shapes_r.append((P, P))
            shapes_t.append((M0, P))
        stack.rnet_list = [np.asmatrix(rl[s, :r * c].reshape(r, c)) for s, (r, c) in enumerate(shapes_r)]
        stack.tnet_list = [np.asmatrix(tl[s, :r * c].reshape(r, c)) for s, (r, c) in enumerate(shapes_t)]
    if not calc_fluxes:
        return
    flags = int(out['flags'][0].item())
    f = out['fluxes'][0].cpu().numpy()
    dn, up = out['vec_coef_lens']
    vd = out['vec_coef_down'][0].cpu().numpy()
    vu = out['vec_coef_up'][0].cpu().numpy()
    offs = np.cumsum([0] + dn)
    stack.vec_coef_down = [np.asmatrix(vd[offs[i]:offs[i + 1]].reshape(-1, 1)) for i in range(len(dn))]
    offs = np.cumsum([0] + up)
    stack.vec_coef_up = [np.asmatrix(vu[offs[i]:offs[i + 1]].reshape(-1, 1)) for i in range(len(up))]
    df = [f[0, 0]] + [complex(f[i, 0], f[i, 1]) for i in range(1, L - 1)]
    up0 = f[L, 0]
    if is_film(sub):
        if flags & _lib.PT_NO_PROP_SUB:
            print("Warning: there are no propagating modes in the semi-inf \n substrate therefore "
                  "cannot calculate energy fluxes here.")
            stack.a_list = np.zeros(L - 2)
            stack.r_list = np.zeros(L - 2)
            stack.t_list = np.zeros(L - 2)
        else:
            stack.a_list = [float(v) for v in out['a_list'][0].cpu().numpy()]
            stack.t_list = [float(v) for v in out['t_list'][0].cpu().numpy()]
            stack.r_list = [float(out['r_list'][0].item())]
            df.append(f[L - 1, 0])
    else:
        # substrate is nanostructured: lists over the air-gap fluxes only
        # (backend/stack.py:402-426)
        a_list, t_list = [], []
        for i in range(1, len(df) - 1):
            a_list.append(abs(abs(df[i]) - abs(df[i + 1])))
        a_list.append(abs(df[0] - df[-1] - up0))
        for i in range(0, len(df) - 2):
            t_list.append(abs(df[i + 2]) / abs(df[i]))
        t_list.append(abs(df[-1] / df[0]))
        stack.a_list, stack.t_list, stack.r_list = a_list, t_list, [abs(up0 / df[0])]
    stack.down_fluxes = df
    stack.up_flux = [up0]


# ---------------------------------------------------------------------------
# uneven batch of dense stacks in one launch
# ---------------------------------------------------------------------------

_POINT_DTYPE = np.dtype([
    ('n_layers', np.int32), ('P', np.int32), ('pol', np.int32), ('spec', np.int32),
    ('num_prop', np.int32, 3), ('_pad', np.int32),
    ('layer_off', np.int64), ('inc_off', np.int64), ('rnet_off', np.int64),
    ('tnet_off', np.int64), ('list_off', np.int64), ('flux_off', np.int64),
])
_LAYER_DTYPE = np.dtype([
    ('M', np.int32), ('dense', np.int32), ('R12', np.uint64), ('T12', np.uint64), ('R21', np.uint64),
    ('T21', np.uint64), ('kz', np.uint64), ('height_norm', np.float64),
])
assert _POINT_DTYPE.itemsize == C.sizeof(_lib.EmuStackPoint)
assert _LAYER_DTYPE.itemsize == C.sizeof(_lib.EmuVarLayer)


class VarStack(object):
    """One stack of an uneven dense batch (one spectral point).

    layers: bottom to top, each (R12, T12, R21, T21, dense, kz, height_norm)
    with device tensors of ONE point (film: diagonals [P]; dense: [P, P],
    [M, P], [M, M], [P, M]; kz [M] for finite layers, else None); the
    substrate and the superstrate are films.  pol: a polarisation name, or
    incoming [P] (device) amplitudes.  spec / num_prop (air, superstrate,
    substrate) may be left None and given to ``StackVarSolver.solve`` as
    device tensors.
    """

    __slots__ = ('layers', 'P', 'pol', 'incoming', 'spec', 'num_prop', 'M', 'D', 'cost')

    def __init__(self, layers, P, pol='TE', incoming=None, spec=None, num_prop=None):
        self.layers = layers
        self.P = int(P)
        self.incoming = incoming
        self.pol = _lib.POL_INCOMING if incoming is not None else _lib.POL[pol]
        self.spec = spec
        self.num_prop = num_prop
        self.M = [int(ly[3].shape[-1]) if ly[4] else self.P for ly in layers]
        self.D = max([self.P] + self.M)
        # the one-CTA cascade's work grows as D^3 per layer
        self.cost = float(len(layers)) * self.D ** 3


class StackVarSolver(object):
    """Cascade + fluxes of an uneven batch of dense stacks in one launch
    (emu_stack_var_batch): each stack is the one-CTA path of
    ``DenseStackSolver`` with its own shapes, taken costliest first by a
    persistent kernel."""

    def __init__(self, device=None):
        self.device = device or _dev()
        self._ws = None

    def solve(self, stacks, spec=None, num_prop=None, n_slots=0, ws_budget_bytes=None, want_fluxes=False):
        """Returns a dict of packed device outputs (R_net, T_net [sum P^2],
        a_list, t_list [sum (L-1)], r_list, flags, info [n], fluxes [sum
        2(L+1)] if asked) and the host offsets (rnet_off, list_off,
        flux_off).  spec [n] / num_prop [n, 3] int32 device tensors override
        the stacks' own values."""
        n = len(stacks)
        dev = self.device
        pts = np.zeros(n, _POINT_DTYPE)
        n_lay = sum(len(s.layers) for s in stacks)
        lays = np.zeros(n_lay, _LAYER_DTYPE)
        keep = []
        lo = ro = li = fo = io = 0
        inc_parts = []
        for i, s in enumerate(stacks):
            L, P = len(s.layers), s.P
            p = pts[i]
            p['n_layers'], p['P'], p['pol'] = L, P, s.pol
            if s.spec is not None:
                p['spec'] = int(s.spec)
            if s.num_prop is not None:
                p['num_prop'] = [int(x) for x in s.num_prop]
            p['layer_off'], p['rnet_off'], p['tnet_off'] = lo, ro, ro
            p['list_off'], p['flux_off'] = li, fo
            p['inc_off'] = -1
            if s.incoming is not None:
                p['inc_off'] = io
                inc_parts.append(s.incoming.reshape(-1))
                io += P
            for j, (R12, T12, R21, T21, dense, kz, hn) in enumerate(s.layers):
                e = lays[lo + j]
                e['M'], e['dense'] = s.M[j], int(bool(dense))
                for nm, t in (('R12', R12), ('T12', T12), ('R21', R21), ('T21', T21), ('kz', kz)):
                    if t is not None:
                        if not t.is_cuda or t.dtype != c128 or not t.is_contiguous():
                            raise TypeError('stack %d layer %d %s must be a contiguous CUDA complex128 '
                                            'tensor' % (i, j, nm))
                        e[nm] = t.data_ptr()
                        keep.append(t)
                e['height_norm'] = float(hn)
            lo += L
            ro += P * P
            li += L - 1
            fo += 2 * (L + 1)
        out = {
            'R_net': torch.empty(ro, dtype=c128, device=dev),
            'T_net': torch.empty(ro, dtype=c128, device=dev),
            'a_list': torch.empty(li, dtype=torch.float64, device=dev),
            't_list': torch.empty(li, dtype=torch.float64, device=dev),
            'r_list': torch.empty(n, dtype=torch.float64, device=dev),
            'flags': torch.zeros(n, dtype=torch.int32, device=dev),
            'info': torch.zeros(n, dtype=torch.int32, device=dev),
        }
        if want_fluxes:
            out['fluxes'] = torch.empty(fo, dtype=torch.float64, device=dev)
        order = np.argsort([-s.cost for s in stacks], kind='stable').astype(np.int32)
        h_pts = torch.from_numpy(pts.view(np.uint8)).pin_memory()
        h_lays = torch.from_numpy(lays.view(np.uint8)).pin_memory()
        h_ord = torch.from_numpy(order).pin_memory()
        d_pts = h_pts.to(dev, non_blocking=True)
        d_lays = h_lays.to(dev, non_blocking=True)
        d_ord = h_ord.to(dev, non_blocking=True)
        iv = d_pts.view(torch.int32).view(n, _POINT_DTYPE.itemsize // 4)
        if spec is not None:
            iv[:, 3] = spec.to(torch.int32)
        if num_prop is not None:
            iv[:, 4:7] = num_prop.to(torch.int32)
        inc = torch.cat(inc_parts) if inc_parts else None
        d = _lib.EmuStackVarBatch()
        d.n_stacks = n
        d.d_points, d.d_order, d.d_layers = ptr(d_pts), ptr(d_ord), ptr(d_lays)
        d.n_layer_desc = n_lay
        d.d_incoming, d.incoming_len = ptr(inc), io
        d.d_R_net, d.rnet_len = ptr(out['R_net']), ro
        d.d_T_net, d.tnet_len = ptr(out['T_net']), ro
        d.d_a_list, d.d_t_list, d.list_len = ptr(out['a_list']), ptr(out['t_list']), li
        d.d_fluxes, d.flux_len = ptr(out.get('fluxes')), fo
        d.d_r_list, d.d_flags, d.d_info = ptr(out['r_list']), ptr(out['flags']), ptr(out['info'])
        d.max_P = max(s.P for s in stacks)
        d.max_D = max(s.D for s in stacks)
        d.max_L = max(len(s.layers) for s in stacks)
        L_ = lib()
        d.n_slots = int(n_slots)
        if ws_budget_bytes is not None:
            d.n_slots = 0
            auto = L_.emu_stack_var_slots(C.byref(d))
            per = (L_.emu_stack_var_workspace_size(C.byref(d)) - 256) / max(auto, 1)
            d.n_slots = max(1, min(auto, int(ws_budget_bytes // max(per, 1))))
        nbytes = L_.emu_stack_var_workspace_size(C.byref(d))
        if self._ws is None or self._ws.numel() < nbytes:
            self._ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        check(L_.emu_stack_var_batch(C.byref(d), ptr(self._ws), C.c_size_t(self._ws.numel()), stream_ptr()),
              'emu_stack_var_batch')
        out['_keep'] = (keep, d_pts, d_lays, d_ord, inc, h_pts, h_lays, h_ord)
        out['rnet_off'] = pts['rnet_off']
        out['list_off'] = pts['list_off']
        out['flux_off'] = pts['flux_off']
        out['n_slots'] = int(L_.emu_stack_var_slots(C.byref(d)))
        return out
