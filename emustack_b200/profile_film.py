"""Run the batched thin-film workload on the GPU for profiling.

    python -m emustack_b200.profile_film [--points N] [--steps K]

Solves K batches of N spectral points of the batched thin-film workload
(the same seeded inputs as bench.py) and prints the mean device time per
batch.  Meant to be wrapped by a profiler (e.g. ncu -k regex:film_stack).
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np
import torch

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--points', type=int, default=32768)
    ap.add_argument('--steps', type=int, default=3)
    ap.add_argument('--pol', default='TE')
    args = ap.parse_args()
    from bench import workload, MAX_ORDER, PERIOD, N_FILMS
    from emustack_b200.films import FilmStackSolver
    w = workload(0)
    B = min(args.points, len(w['wl']))
    dev = torch.device('cuda')
    s = FilmStackSolver(N_FILMS + 2, MAX_ORDER, PERIOD)
    d = [torch.tensor(np.ascontiguousarray(w[k][:B]), device=dev) for k in ('wl', 'k_pll', 'n')]
    h = torch.tensor(w['heights'], device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    s.solve(*d, h, pol=args.pol)
    torch.cuda.synchronize()
    ev[0].record()
    for _ in range(args.steps):
        s.solve(*d, h, pol=args.pol)
    ev[1].record()
    torch.cuda.synchronize()
    print('points %d  mean %.3f ms/batch' % (B, ev[0].elapsed_time(ev[1]) / args.steps))


if __name__ == '__main__':
    main()
