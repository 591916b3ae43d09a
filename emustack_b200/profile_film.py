"""Run the batched thin-film workload on the GPU for profiling.

    python -m emustack_b200.profile_film [--points N] [--steps K] [--variant V | --sweep]

Solves K batches of N spectral points of the batched thin-film workload
(the same seeded inputs as bench.py) and prints the mean device time per
batch: with the autotuner's launch variant, a fixed one (--variant), or
each variant in turn (--sweep).  Meant to be wrapped by a profiler (e.g.
ncu -k regex:film_stack).
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
    ap.add_argument('--variant', type=int, default=None)
    ap.add_argument('--sweep', action='store_true')
    args = ap.parse_args()
    from bench import workload, MAX_ORDER, PERIOD, N_FILMS
    from emustack_b200 import _lib
    from emustack_b200.films import FilmStackSolver
    w = workload(0)
    B = min(args.points, len(w['wl']))
    dev = torch.device('cuda')
    s = FilmStackSolver(N_FILMS + 2, MAX_ORDER, PERIOD)
    d = [torch.tensor(np.ascontiguousarray(w[k][:B]), device=dev) for k in ('wl', 'k_pll', 'n')]
    h = torch.tensor(w['heights'], device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for v in (_lib.FILM_VARIANTS if args.sweep else (args.variant,)):
        for _ in range(3):
            s.solve(*d, h, pol=args.pol, variant=v)
        torch.cuda.synchronize()
        ev[0].record()
        for _ in range(args.steps):
            s.solve(*d, h, pol=args.pol, variant=v)
        ev[1].record()
        torch.cuda.synchronize()
        ms = ev[0].elapsed_time(ev[1]) / args.steps
        print('points %d  pol %s  variant %s  mean %.3f ms/batch  %.2fM points/s'
              % (B, args.pol, 'auto' if v is None else v, ms, B / ms / 1e3))


if __name__ == '__main__':
    main()
