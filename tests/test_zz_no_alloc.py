"""The allocation-free film solve (emu_film_stack_batch_noalloc).

Some callers cannot allocate device memory at the point where they solve:
a host thread inside a latency-critical loop (cudaMalloc and cudaFree
synchronise the whole device), code that runs while another framework's
caching allocator owns the device heap, or an embedding that must not fail
on memory pressure once it has started.  For them the film solve can use a
fixed scratch array compiled into the library instead of a workspace the
caller allocates.  Only incoming amplitudes (pol 'incoming', any order may
carry light) need that scratch; the standard polarisations use none.

The tests call the entry point through the C ABI twice in a row with
different shapes and inputs, so the second call runs over whatever the
first left in the shared array, and check each result against the CPU
oracle (a restatement of the reference's FP64 algorithm) and against the
workspace entry point emu_film_stack_batch, at the tolerance of the other
film tests.  The file is collected last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = dict(rtol=1e-9, atol=1e-10)


def _inputs(seed, B, L, P=None):
    from oracle.gsm_oracle import k_parallel_from_angles
    rng = np.random.default_rng(seed)
    n = np.concatenate([[1.46 + 0j], rng.uniform(1.3, 4.0, L - 2) + 1j * rng.uniform(0, 0.5, L - 2),
                        [1.0 + 0j]])
    h = rng.uniform(20, 300, L - 2)
    wl = rng.uniform(350, 1100, B)
    kp = np.array([k_parallel_from_angles(w, t, f) for w, t, f in
                   zip(wl, rng.uniform(0, 60, B), rng.uniform(0, 90, B))])
    inc = None
    if P is not None:
        # several non-zero amplitudes per point, in propagating and evanescent orders
        inc = np.zeros((B, P), complex)
        for b in range(B):
            idx = rng.choice(P, size=6, replace=False)
            inc[b, idx] = rng.standard_normal(6) + 1j * rng.standard_normal(6)
    return wl, kp, np.tile(n, (B, 1)), h, inc


def _entry():
    from emustack_b200 import _lib
    L_ = _lib.lib()
    f = L_.emu_film_stack_batch_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(_lib.EmuFilmStackBatch), C.c_void_p]
    L_.emu_film_stack_static_scratch_bytes.restype = C.c_size_t
    L_.emu_film_stack_workspace_size.restype = C.c_size_t
    return L_, f


def _run_noalloc(L, max_order, wl, kp, n, h, pol, inc):
    """One call of the allocation-free entry point; returns host outputs
    and the workspace bytes the request would have needed."""
    from emustack_b200 import _lib
    from emustack_b200.films import FilmStackSolver
    L_, f = _entry()
    dev = torch.device('cuda')
    args = [torch.tensor(wl, device=dev), torch.tensor(kp, device=dev), torch.tensor(n, device=dev),
            torch.tensor(h, device=dev)]
    d_inc = None if inc is None else torch.tensor(inc, device=dev)
    s = FilmStackSolver(L, max_order, 500.0)
    out = s.outputs(len(wl))
    for k, v in out.items():
        v.fill_(float('nan') if (v.is_floating_point() or v.is_complex()) else 0)
    d = s.descriptor(args[0], args[1], args[2], args[3], pol, d_inc, None, out)
    need = L_.emu_film_stack_workspace_size(C.byref(d))
    st = f(C.byref(d), _lib.stream_ptr())
    assert st == 0, _lib.STATUS_NAMES.get(st, st)
    torch.cuda.synchronize()
    res = {k: v.cpu().numpy().copy() for k, v in out.items()}
    # the workspace entry point on the same inputs
    ref = FilmStackSolver(L, max_order, 500.0).solve(*args, pol=pol, incoming=d_inc)
    torch.cuda.synchronize()
    ref = {k: v.cpu().numpy().copy() for k, v in ref.items()}
    return res, ref, need, s.npw


def _check_against_oracle(res, wl, kp, n, h, max_order, pol, inc, pts, tag):
    from oracle import gsm_oracle as O
    npw = res['R_net'].shape[1] // 2
    for b in pts:
        r = O.film_stack_point(n[b], h, wl[b], kp[b], 500.0, max_order=max_order, pol=pol,
                               incoming_amplitudes=None if inc is None else inc[b])
        np.testing.assert_allclose(res['R_net'][b], np.diag(r.R_net), **TOL, err_msg='%s p%d R' % (tag, b))
        np.testing.assert_allclose(res['T_net'][b], np.diag(r.T_net), **TOL, err_msg='%s p%d T' % (tag, b))
        np.testing.assert_allclose(res['a_list'][b], np.asarray(r.a_list, float), rtol=1e-9, atol=1e-9,
                                   err_msg='%s p%d a' % (tag, b))
        np.testing.assert_allclose(res['t_list'][b], np.asarray(r.t_list, float), rtol=1e-9, atol=1e-9,
                                   err_msg='%s p%d t' % (tag, b))
        assert res['R_net'].shape[1] == 2 * npw


def test_noalloc_incoming_amplitudes_use_the_scratch_twice():
    """Two back-to-back calls with incoming amplitudes (the polarisation
    that reads and writes the scratch array), of different shapes, each
    checked against the oracle and against the workspace entry point."""
    L_, _ = _entry()
    cap = L_.emu_film_stack_static_scratch_bytes()
    calls = [(21, 96, 12, 5), (22, 150, 7, 4)]   # seed, points, layers, max order (Npw 81, 49)
    for call, (seed, B, L, mo) in enumerate(calls):
        from emustack_b200.films import grating_orders
        P = 2 * len(grating_orders(mo, 500.0, 500.0, False)[0])
        wl, kp, n, h, inc = _inputs(seed, B, L, P)
        res, ref, need, npw = _run_noalloc(L, mo, wl, kp, n, h, 'incoming', inc)
        assert 0 < need <= cap
        for k in ('R_net', 'T_net', 'a_list', 't_list', 'r_list'):
            np.testing.assert_allclose(res[k], ref[k], **TOL, err_msg='call %d %s' % (call, k))
        assert np.array_equal(res['flags'], ref['flags'])
        _check_against_oracle(res, wl, kp, n, h, mo, 'TE', inc, range(0, B, max(1, B // 5)),
                              'call %d' % call)


def test_noalloc_standard_polarisations_need_no_scratch():
    """TE and R Circ keep their flux-pass scalars in shared memory: the
    request needs no workspace, and the results equal the oracle's."""
    for call, (seed, B, pol) in enumerate(((11, 300, 'TE'), (12, 517, 'R Circ'))):
        wl, kp, n, h, _ = _inputs(seed, B, 8)
        res, ref, need, _ = _run_noalloc(8, 4, wl, kp, n, h, pol, None)
        assert need == 0
        for k in ('R_net', 'T_net', 'a_list', 't_list', 'r_list'):
            np.testing.assert_allclose(res[k], ref[k], **TOL, err_msg='call %d %s' % (call, k))
        _check_against_oracle(res, wl, kp, n, h, 4, pol, None, (0, B - 1), 'call %d' % call)


def test_noalloc_rejects_requests_above_the_scratch_size():
    from emustack_b200 import _lib
    from emustack_b200.films import FilmStackSolver
    L_, f = _entry()
    cap = L_.emu_film_stack_static_scratch_bytes()
    L, mo = 12, 5
    s = FilmStackSolver(L, mo, 500.0)
    per_point = s.npw * L * 2 * 5 * 16
    B = cap // per_point + 1
    wl, kp, n, h, inc = _inputs(13, B, L, s.P)
    dev = torch.device('cuda')
    args = [torch.tensor(wl, device=dev), torch.tensor(kp, device=dev), torch.tensor(n, device=dev),
            torch.tensor(h, device=dev)]
    out = s.outputs(B)
    d = s.descriptor(args[0], args[1], args[2], args[3], 'incoming', torch.tensor(inc, device=dev),
                     None, out)
    assert L_.emu_film_stack_workspace_size(C.byref(d)) > cap
    assert f(C.byref(d), _lib.stream_ptr()) == 5  # EMU_E_WORKSPACE
