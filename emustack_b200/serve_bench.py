"""Open-loop Poisson-arrival load test of the continuous-batching server.

    python -m emustack_b200.serve_bench [--rates 1000,10000,100000] [--seconds 2]
                                        [--batching mixed|grouped] [--max-batch N]

Requests are all-film spectral points whose sizes follow the uneven-batch
distribution: plane-wave count P = 2 Npw log-uniform in [50, 900] (the
order set of the max order whose Npw is nearest, period 500 nm), 2-12
finite layers, n U(1.3, 4.0) + i U(0, 0.5) on n = 1.46 under air, thickness
U(20, 300) nm, wavelength U(350, 1100) nm, theta U(0, 60), phi U(0, 90) deg,
polarisation cycling TE / TM / un / R Circ.  Arrival times are drawn in
advance (exponential gaps at the offered rate); a submitter thread hands
each request to the server at its arrival time and latency is measured from
that scheduled time (so a slow submitter cannot hide queueing).  One JSON
line per rate: offered and achieved throughput, p50 / p99 latency, batches.

With --array-frac F a fraction F of the requests are array stacks
(``ArrayRequest``): a film substrate (n = 1.46), 2-12 finite layers each a
film or one of the nanostructured layers of the request's spectral point,
and air.  Spectral points come from a pool (--array-pool of them, P log-
uniform in [50, 900] like the films, M = P + 20 Bloch modes, two array
layers per point with synthetic J, J_dag complex N(0, 1)/sqrt(P) made on the
device and Bloch k_z Re U(0, 2 k0), Im U(0, 0.1 k0)), so requests share
layers as a sweep over heights and layer orders does; the server computes
each layer's interface once and serves the rest from its device cache.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import sys
import threading
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def order_table(period, max_mo=16):
    from emustack_b200.films import grating_orders
    return np.array([len(grating_orders(m, period, period)[0]) for m in range(max_mo + 1)])


def make_requests(n, seed=0, period=500.0):
    from emustack_b200.serving import FilmRequest
    rng = np.random.default_rng(seed)
    tab = order_table(period)
    pols = ('TE', 'TM', 'un', 'R Circ')
    reqs = []
    P = np.exp(rng.uniform(np.log(50), np.log(900), n))
    for i in range(n):
        mo = int(np.argmin(np.abs(tab - P[i] / 2)))
        L = int(rng.integers(2, 13)) + 2
        nn = np.concatenate([[1.46 + 0j], rng.uniform(1.3, 4.0, L - 2) + 1j * rng.uniform(0, 0.5, L - 2),
                             [1.0 + 0j]])
        wl = rng.uniform(350, 1100)
        th, ph = np.radians(rng.uniform(0, 60)), np.radians(rng.uniform(0, 90))
        k = 2 * np.pi / wl
        kp = np.array([k * np.sin(th) * np.cos(ph), k * np.sin(th) * np.sin(ph)])
        reqs.append(FilmRequest(nn, rng.uniform(20, 300, L - 2), wl, kp, period, mo, pol=pols[i % 4]))
    return reqs


def make_array_pool(n_points, seed=0, period=500.0, device='cuda'):
    """Spectral points with two synthetic array layers each."""
    import torch
    from emustack_b200.array_serving import ArrayLayer
    rng = np.random.default_rng(seed)
    tab = order_table(period)
    g = torch.Generator(device=device).manual_seed(seed)
    pool = []
    for i in range(n_points):
        P = float(np.exp(rng.uniform(np.log(50), np.log(900))))
        mo = int(np.argmin(np.abs(tab - P / 2)))
        P = 2 * int(tab[mo])
        M = P + 20
        wl = float(rng.uniform(350, 1100))
        th, ph = np.radians(rng.uniform(0, 60)), np.radians(rng.uniform(0, 90))
        k = 2 * np.pi / wl
        kp = np.array([k * np.sin(th) * np.cos(ph), k * np.sin(th) * np.sin(ph)])
        k0 = 2 * np.pi / (wl / period)
        cr = lambda *sh: torch.complex(torch.randn(sh, dtype=torch.float64, device=device, generator=g),
                                       torch.randn(sh, dtype=torch.float64, device=device, generator=g))
        lays = []
        for _ in range(2):
            kz = rng.uniform(0, 2, M) * k0 + 1j * rng.uniform(0, 0.1, M) * k0
            lays.append(ArrayLayer(kz, J=cr(P, M) / np.sqrt(P), J_dag=cr(M, P) / np.sqrt(P)))
        pool.append((mo, wl, kp, lays))
    return pool


def make_array_requests(n, pool, seed=0, period=500.0):
    from emustack_b200.array_serving import ArrayRequest
    rng = np.random.default_rng(seed)
    pols = ('TE', 'TM', 'un', 'R Circ')
    reqs = []
    for i in range(n):
        mo, wl, kp, lays = pool[int(rng.integers(len(pool)))]
        K = int(rng.integers(2, 13))
        mid = [lays[int(rng.integers(2))] if rng.random() < 0.5
               else complex(rng.uniform(1.3, 4.0), rng.uniform(0, 0.5)) for _ in range(K)]
        reqs.append(ArrayRequest([1.46 + 0j] + mid + [1.0 + 0j], rng.uniform(20, 300, K), wl, kp, period, mo,
                                 pol=pols[i % 4]))
    return reqs


def mixed_requests(n, seed, array_frac, pool):
    """n requests, a fraction array_frac of them array stacks, in random order."""
    na = int(round(n * array_frac)) if pool else 0
    reqs = make_requests(n - na, seed) + (make_array_requests(na, pool, seed + 7) if na else [])
    order = np.random.default_rng(seed + 3).permutation(len(reqs))
    return [reqs[i] for i in order]


def run_rate(rate, seconds, batching, max_batch, seed, array_frac=0.0, pool=None, n_streams=2):
    import torch
    from emustack_b200.serving import GsmServer
    n = max(int(rate * seconds), 200)
    reqs = mixed_requests(n, seed, array_frac, pool)
    rng = np.random.default_rng(seed + 1)
    gaps = rng.exponential(1.0 / rate, n)
    srv = GsmServer(max_batch=max_batch, batching=batching, n_streams=n_streams).start()
    # warm the server: bursts as large as the batches this rate will form, so
    # that staging and device buffers have grown before the timed run
    burst = mixed_requests(max(64, min(max_batch, int(rate * 0.2))), seed + 2, array_frac, pool)
    for _ in range(2):
        for f in [srv.submit(r) for r in burst]:
            f.result(timeout=300)
    srv.latencies.clear()
    srv.array_latencies.clear()
    c = srv.cache
    c.hits = c.misses = c.evictions = 0
    srv.batch_sizes.clear()
    srv.n_batches = 0
    srv.t_first = srv.t_last = None
    for k in srv.prof:
        srv.prof[k] = 0.0
    t0 = time.perf_counter() + 0.05
    arrivals = t0 + np.cumsum(gaps)
    futs = []

    def submitter():
        # hands over every request whose arrival time has passed, then sleeps
        # (releasing the interpreter lock) until the next arrival, at least
        # `tick`: requests reach the server in small bursts, and the delay
        # counts in their latency (measured from the scheduled arrival)
        tick = 2e-4
        i = 0
        while i < n:
            now = time.perf_counter()
            while i < n and arrivals[i] <= now:
                reqs[i].t_arrival = float(arrivals[i])
                futs.append(srv.submit(reqs[i]))
                i += 1
            if i < n:
                time.sleep(max(tick, arrivals[i] - time.perf_counter()))

    # a server process keeps the cyclic garbage collector out of the request
    # path (a full collection over ~1e5 live request objects takes tens of ms)
    gc.collect()
    gc.disable()
    try:
        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        for f in futs:
            f.result(timeout=300)
    finally:
        gc.enable()
    srv.stop()
    st = srv.stats()
    torch.cuda.synchronize()
    out = {
        'offered_per_s': rate, 'requests': n, 'batching': batching, 'max_batch': max_batch,
        'streams': n_streams,
        'achieved_per_s': st['throughput_per_s'], 'p50_ms': st['p50_ms'], 'p99_ms': st['p99_ms'],
        'batches': st['batches'], 'mean_batch': st['mean_batch'],
        'host_ms_per_batch': {k[:-2]: 1e3 * v / max(st['batches'], 1) for k, v in srv.prof.items()},
        'mean_P': float(np.mean([2 * r.npw for r in reqs])),
        'mean_layers': float(np.mean([len(r.layers) if hasattr(r, 'air_key') else len(r.n) for r in reqs])),
    }
    if array_frac:
        c = st['smatrix_cache']
        out.update(array_frac=array_frac, array_requests=st['array_requests'],
                   array_p50_ms=st['array_p50_ms'], array_p99_ms=st['array_p99_ms'],
                   cache_hits=c['hits'], cache_misses=c['misses'], cache_entries=c['entries'],
                   cache_gb=c['bytes'] / 1e9)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--rates', default='1000,3000,10000,30000,100000')
    ap.add_argument('--seconds', type=float, default=2.0)
    ap.add_argument('--batching', default='mixed')
    ap.add_argument('--max-batch', type=int, default=32768)
    ap.add_argument('--seed', type=int, default=0)
    ap.add_argument('--array-frac', type=float, default=0.0, help='fraction of array-stack requests')
    ap.add_argument('--array-pool', type=int, default=32, help='spectral points of the array layers')
    ap.add_argument('--streams', type=int, default=2, help='batches in flight at once')
    args = ap.parse_args()
    pool = make_array_pool(args.array_pool, args.seed + 11) if args.array_frac > 0 else None
    for r in [float(x) for x in args.rates.split(',')]:
        print(json.dumps(run_rate(r, args.seconds, args.batching, args.max_batch, args.seed,
                                  args.array_frac, pool, args.streams)), flush=True)


if __name__ == '__main__':
    main()
