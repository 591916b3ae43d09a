"""Replica sharding over spectral points with world_size 2 on the gloo
backend (CPU): shards cover every point once, and the gathered per-point
results equal a single-process run.  The per-rank solve here is the CPU
oracle on a few thin-film points (the GPU solve is covered by -m gpu)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from emustack_b200.replicas import shard_bounds


def test_shard_bounds_cover_all_points():
    for n in (0, 1, 7, 32768, 32769):
        for w in (1, 2, 3, 8):
            seen = []
            for r in range(w):
                s, e = shard_bounds(n, r, w)
                seen.extend(range(s, e))
                assert e - s in (n // w, n // w + 1)
            assert seen == list(range(n))


def _points():
    from oracle.gsm_oracle import k_parallel_from_angles
    rng = np.random.default_rng(3)
    B = 7
    wl = rng.uniform(400, 900, B)
    kp = np.array([k_parallel_from_angles(w, t, 10.0) for w, t in zip(wl, rng.uniform(0, 50, B))])
    return wl, kp


def _solve(wl, kp):
    from oracle import gsm_oracle as O
    nl = np.array([1.5 + 0j, 2.2 + 0.05j, 1.0 + 0j])
    a, r = [], []
    for w, k in zip(wl, kp):
        res = O.film_stack_point(nl, [110.0], w, k, 450.0, max_order=1, pol='TE')
        a.append(np.asarray(res.a_list, float))
        r.append(float(res.r_list[0]))
    return {'a_list': np.array(a), 'r_list': np.array(r)}


def _worker(rank, world, port, out_q):
    import torch.distributed as dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    from emustack_b200.replicas import gather_results, shard
    wl, kp = _points()
    (wl_s, kp_s), _ = shard([wl, kp], rank, world)
    res = gather_results(_solve(wl_s, kp_s), len(wl))
    if rank == 0:
        out_q.put(res)
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_gloo_matches_single_process():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    wl, kp = _points()
    ref = _solve(wl, kp)
    np.testing.assert_array_equal(res['a_list'], ref['a_list'])
    np.testing.assert_array_equal(res['r_list'], ref['r_list'])
