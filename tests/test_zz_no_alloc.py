"""The allocation-free film solve (emu_film_stack_batch_noalloc).

It serves callers that must not allocate device memory where they solve
(cudaMalloc / cudaFree synchronise the device and can fail under memory
pressure; another framework's caching allocator may own the heap): the
solve uses a fixed scratch array built into the library instead of a
caller workspace.  This test calls it through the C ABI, twice in a row on
different inputs, and checks each result against the workspace entry point
emu_film_stack_batch on the same inputs, at the tolerance of the other film
tests.  It lives in its own file, collected last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = dict(rtol=1e-9, atol=1e-10)


def _inputs(seed, B, L):
    from oracle.gsm_oracle import k_parallel_from_angles
    rng = np.random.default_rng(seed)
    n = np.concatenate([[1.46 + 0j], rng.uniform(1.3, 4.0, L - 2) + 1j * rng.uniform(0, 0.5, L - 2),
                        [1.0 + 0j]])
    h = rng.uniform(20, 300, L - 2)
    wl = rng.uniform(350, 1100, B)
    kp = np.array([k_parallel_from_angles(w, t, f) for w, t, f in
                   zip(wl, rng.uniform(0, 60, B), rng.uniform(0, 90, B))])
    return wl, kp, np.tile(n, (B, 1)), h


def test_noalloc_matches_workspace_entry_point_twice():
    from emustack_b200 import _lib
    from emustack_b200.films import FilmStackSolver
    L_ = _lib.lib()
    f = L_.emu_film_stack_batch_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(_lib.EmuFilmStackBatch), C.c_void_p]
    L_.emu_film_stack_static_scratch_bytes.restype = C.c_size_t
    cap = L_.emu_film_stack_static_scratch_bytes()
    assert cap > 0
    dev = torch.device('cuda')
    L = 8
    for call, (seed, B, pol) in enumerate(((11, 300, 'TE'), (12, 517, 'R Circ'))):
        wl, kp, n, h = _inputs(seed, B, L)
        args = [torch.tensor(wl, device=dev), torch.tensor(kp, device=dev),
                torch.tensor(n, device=dev), torch.tensor(h, device=dev)]
        # reference result: the workspace entry point
        ref_solver = FilmStackSolver(L, 4, 500.0)
        ref = {k: v.clone() for k, v in ref_solver.solve(*args, pol=pol).items()}
        # allocation-free entry point, outputs in separate buffers
        s = FilmStackSolver(L, 4, 500.0)
        out = {k: torch.full_like(v, float('nan')) if v.is_floating_point() or v.is_complex()
               else torch.zeros_like(v) for k, v in ref.items()}
        d = s.descriptor(args[0], args[1], args[2], args[3], pol, None, None, out)
        assert L_.emu_film_stack_workspace_size(C.byref(d)) <= cap
        st = f(C.byref(d), _lib.stream_ptr())
        assert st == 0, _lib.STATUS_NAMES.get(st, st)
        torch.cuda.synchronize()
        for k in ('R_net', 'T_net', 'a_list', 't_list', 'r_list'):
            np.testing.assert_allclose(out[k].cpu().numpy(), ref[k].cpu().numpy(), **TOL,
                                       err_msg='call %d %s' % (call, k))
        assert torch.equal(out['flags'], ref['flags'])


def test_noalloc_rejects_requests_above_the_scratch_size():
    from emustack_b200 import _lib
    from emustack_b200.films import FilmStackSolver
    L_ = _lib.lib()
    f = L_.emu_film_stack_batch_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(_lib.EmuFilmStackBatch), C.c_void_p]
    L_.emu_film_stack_static_scratch_bytes.restype = C.c_size_t
    cap = L_.emu_film_stack_static_scratch_bytes()
    L = 12
    per_point = L * 2 * 5 * 16
    B = cap // per_point + 1
    wl, kp, n, h = _inputs(13, B, L)
    dev = torch.device('cuda')
    args = [torch.tensor(wl, device=dev), torch.tensor(kp, device=dev), torch.tensor(n, device=dev),
            torch.tensor(h, device=dev)]
    s = FilmStackSolver(L, 1, 500.0)
    out = s.outputs(B)
    d = s.descriptor(args[0], args[1], args[2], args[3], 'TE', None, None, out)
    assert L_.emu_film_stack_workspace_size(C.byref(d)) > cap
    assert f(C.byref(d), _lib.stream_ptr()) == 5  # EMU_E_WORKSPACE
