"""Host-side logic of array-stack requests (no GPU): the layer interface
cache's LRU accounting, the per-point workspace estimate against the
library's own emu_stack_dense_workspace_size, and request validation."""
import ctypes as C

import numpy as np
import pytest


class _E(object):
    def __init__(self, nbytes):
        self.nbytes = nbytes
        self.users = 0


def test_smatrix_cache_lru_and_pinning():
    from emustack_b200.array_serving import SMatrixCache
    c = SMatrixCache(100)
    a, b, d = _E(40), _E(40), _E(40)
    c.put('a', a)
    c.put('b', b)
    assert c.get('a') is a                     # a is now the most recent
    c.put('d', d)                              # 120 > 100: evicts b (least recent)
    assert 'b' not in c.entries and c.bytes == 80 and c.evictions == 1
    assert c.get('b') is None
    a.users = d.users = 1                      # in use by batches in flight
    e = _E(40)
    e.users = 1                                # new entries are pinned by their batch
    c.put('e', e)
    assert c.bytes == 120 and set(c.entries) == {'a', 'd', 'e'}
    a.users = 0
    c.evict()                                  # a is the oldest unpinned
    assert set(c.entries) == {'d', 'e'} and c.bytes == 80
    c.drop('d')
    assert c.bytes == 40
    s = c.stats()
    assert s['hits'] == 1 and s['misses'] == 1 and s['entries'] == 1


@pytest.mark.parametrize('P,Ms', [(26, [26, 40, 26]), (58, [58, 60, 64, 58, 58]),
                                  (98, [98, 100, 98]), (634, [634, 700, 660, 634])])
def test_workspace_estimate_matches_library(P, Ms):
    from emustack_b200 import _lib
    from emustack_b200.array_serving import dense_workspace_bytes
    L = len(Ms)
    arr = (_lib.EmuLayer * L)()
    for i, M in enumerate(Ms):
        arr[i].M = M
        arr[i].dense = int(M != P or 0 < i < L - 1)
        for nm in ('d_R12', 'd_T12', 'd_R21', 'd_T21', 'd_kz'):
            setattr(arr[i], nm, 16)            # non-null; sizes only, never dereferenced
    d = _lib.EmuStackDense()
    d.batch, d.n_layers, d.P = 1, L, P
    d.h_layers = C.cast(arr, C.POINTER(_lib.EmuLayer))
    d.d_R_net = d.d_T_net = 16
    got = _lib.lib().emu_stack_dense_workspace_size(C.byref(d))
    assert got == dense_workspace_bytes(P, Ms) + 256


def test_array_request_validation_and_signature():
    from emustack_b200.array_serving import ArrayLayer, ArrayRequest
    from emustack_b200.films import grating_orders
    P = 2 * len(grating_orders(2, 500.0)[0])
    rng = np.random.default_rng(0)
    M = P + 4
    ly = ArrayLayer(rng.normal(size=M) + 0j, J=np.zeros((P, M)), J_dag=np.zeros((M, P)))
    r = ArrayRequest([1.46, ly, 2.0 + 0.1j, 1.0], [100.0, 50.0], 600.0, [0.001, 0.0], 500.0, 2, pol='TM')
    assert r.signature == ('array', 2, 500.0, 500.0, False, 'TM', (0, M, 0, 0))
    assert r.bytes_on_device() > ly.smatrix_bytes()
    assert r.wl_norm() == 600.0 / 500.0
    r2 = ArrayRequest([1.46, ly, 1.0], [100.0], 1000.0, [0.0, 0.0], 500.0, 2)
    assert r2.wl_norm() == 2.0 + 1e-10           # exact multiple nudged as the reference does
    with pytest.raises(ValueError):
        ArrayRequest([1.46, ly, 1.0], [100.0, 3.0], 600.0, [0, 0], 500.0, 2)
    with pytest.raises(ValueError):              # order set of max order 3 has more plane waves
        ArrayRequest([1.46, ly, 1.0], [100.0], 600.0, [0, 0], 500.0, 3)
    with pytest.raises(NotImplementedError):
        ArrayRequest([ly, 1.0], [], 600.0, [0, 0], 500.0, 2)
    with pytest.raises(NotImplementedError):
        ArrayRequest([1.46, ly, 1.0], [100.0], 600.0, [0, 0], 500.0, 2, pol='XY')
    with pytest.raises(ValueError):
        ArrayLayer(np.ones(M), J=np.zeros((P, M)))
    with pytest.raises(ValueError):
        ArrayLayer(np.ones(M), J=np.zeros((P, M + 1)), J_dag=np.zeros((M, P)))
    inc = np.zeros(P, complex)
    inc[3] = 1
    r3 = ArrayRequest([1.46, ly, 1.0], [100.0], 600.0, [0, 0], 500.0, 2, incoming=inc)
    assert r3.pol == 'incoming' and r3.signature[5] == 'incoming'


def test_failed_launch_releases_pinned_entries():
    """A batch whose launch raises after pinning cache entries gives them back,
    so the cache can evict them again."""
    from emustack_b200.array_serving import ArrayBatcher, SMatrixCache
    cache = SMatrixCache(100)
    batcher = ArrayBatcher('cpu', cache)
    a, b = _E(60), _E(60)
    a.users = b.users = 1
    cache.put('a', a)
    cache.put('b', b)
    assert cache.bytes == 120                       # both pinned: over capacity
    batcher._unpin([a, b])
    assert a.users == 0 and b.users == 0 and cache.bytes <= 100
