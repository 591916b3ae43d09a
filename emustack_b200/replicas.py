"""Replica parallelism over spectral points (one process per GPU).

Every (wavelength, angle, stack) solve is independent; the reference
parallelises exactly this way with ``multiprocessing.Pool.map`` over
wavelengths (tests/test_case_0_thin_film_multistack.py:98-102).  Here each
rank of a ``torch.distributed`` group takes a contiguous shard of the point
list, solves it on its own GPU with no collective on the data path, and the
host gathers the per-point results in the original order.
"""
from __future__ import annotations

import numpy as np


def shard_bounds(n_points, rank, world):
    """[start, stop) of rank's contiguous shard; shard sizes differ by <= 1."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError('bad rank / world size')
    base, extra = divmod(int(n_points), int(world))
    start = rank * base + min(rank, extra)
    stop = start + base + (1 if rank < extra else 0)
    return start, stop


def shard(arrays, rank, world):
    """Slice every array's leading axis to rank's shard."""
    n = len(arrays[0])
    s, e = shard_bounds(n, rank, world)
    return [a[s:e] for a in arrays], (s, e)


def gather_results(local, n_points, group=None):
    """All-gather per-point host results (dict of numpy arrays with a leading
    point axis) from every rank and reassemble them in point order.  Uses
    torch.distributed object collectives (host side, any backend)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    parts = [None] * world
    dist.all_gather_object(parts, local, group=group)
    out = {}
    for k in local:
        out[k] = np.concatenate([p[k] for p in parts], axis=0)
        if out[k].shape[0] != n_points:
            raise RuntimeError('gathered %d points, expected %d' % (out[k].shape[0], n_points))
    return out
