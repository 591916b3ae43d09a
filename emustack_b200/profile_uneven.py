"""Time an uneven batch of all-film solves in one launch against per-solve
and per-shape launches.

    python -m emustack_b200.profile_uneven [--points 4096] [--steps 5]

The batch follows the uneven-batch distribution (the film half of it):
P = 2 Npw log-uniform in [50, 900] (the order set of the max order whose Npw
is nearest, period 500 nm), 2-12 finite layers, random indices, heights,
wavelengths and angles (emustack_b200.serve_bench.make_requests).  Prints
one JSON line with points/s for
  * one ``emu_film_var_batch`` launch over the whole batch (device-resident
    inputs, packed by ``FilmVarSolver.plan`` outside the timed region);
  * the same points grouped by shape, one ``emu_film_stack_batch`` launch
    per group;
  * one ``emu_film_stack_batch`` launch per point (the per-solve FP64
    launches the reference's one-call-per-solve structure maps to).
All on one stream, CUDA events, after warm-up.
"""
from __future__ import annotations

import argparse
import collections
import json
import os
import sys

import numpy as np
import torch

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--points', type=int, default=4096)
    ap.add_argument('--steps', type=int, default=5)
    ap.add_argument('--per-solve', type=int, default=512, help='points timed one launch each')
    args = ap.parse_args()
    from emustack_b200.films import FilmStackSolver, FilmVarSolver
    from emustack_b200.serve_bench import make_requests
    dev = torch.device('cuda')
    reqs = make_requests(args.points, seed=0)
    ev = lambda: torch.cuda.Event(enable_timing=True)

    # one uneven launch
    vs = FilmVarSolver(dev)
    pl = vs.plan(reqs)
    vs.solve(pl)
    torch.cuda.synchronize()
    # each timed solve re-copies the packed inputs (~0.2 KB per point) from
    # pinned staging, then launches once
    a, b = ev(), ev()
    vs.solve(pl)
    torch.cuda.synchronize()
    a.record()
    for _ in range(args.steps):
        vs.solve(pl)
    b.record()
    torch.cuda.synchronize()
    ms_var = a.elapsed_time(b) / args.steps

    # grouped by shape: one uniform launch per group
    groups = collections.defaultdict(list)
    for r in reqs:
        groups[(len(r.n), r.max_order, r.pol)].append(r)
    prepared = []
    for (L, mo, pol), rs in groups.items():
        s = FilmStackSolver(L, mo, 500.0, device=dev)
        wl = torch.tensor([r.wl_nm for r in rs], dtype=torch.float64, device=dev)
        kp = torch.tensor(np.stack([r.k_pll for r in rs]), dtype=torch.float64, device=dev)
        n = torch.tensor(np.stack([r.n for r in rs]), dtype=torch.complex128, device=dev)
        h = torch.tensor(np.stack([r.heights for r in rs]), dtype=torch.float64, device=dev)
        prepared.append((s, wl, kp, n, h, pol))
    for s, wl, kp, n, h, pol in prepared:
        s.solve(wl, kp, n, h, pol=pol)
    torch.cuda.synchronize()
    a, b = ev(), ev()
    a.record()
    for _ in range(args.steps):
        for s, wl, kp, n, h, pol in prepared:
            s.solve(wl, kp, n, h, pol=pol)
    b.record()
    torch.cuda.synchronize()
    ms_grouped = a.elapsed_time(b) / args.steps

    # one launch per point (first per_solve points)
    npt = min(args.per_solve, len(reqs))
    single = []
    for r in reqs[:npt]:
        L = len(r.n)
        s = FilmStackSolver(L, r.max_order, 500.0, device=dev)
        single.append((s, torch.tensor([r.wl_nm], dtype=torch.float64, device=dev),
                       torch.tensor(r.k_pll.reshape(1, 2), dtype=torch.float64, device=dev),
                       torch.tensor(r.n.reshape(1, L), dtype=torch.complex128, device=dev),
                       torch.tensor(r.heights, dtype=torch.float64, device=dev), r.pol))
    for s, wl, kp, n, h, pol in single:
        s.solve(wl, kp, n, h, pol=pol)
    torch.cuda.synchronize()
    a, b = ev(), ev()
    a.record()
    for s, wl, kp, n, h, pol in single:
        s.solve(wl, kp, n, h, pol=pol)
    b.record()
    torch.cuda.synchronize()
    ms_single = a.elapsed_time(b) / npt * len(reqs)
    P = np.array([2 * r.npw for r in reqs])
    Ls = np.array([len(r.n) for r in reqs])
    print(json.dumps({
        'points': len(reqs), 'mean_P': float(P.mean()), 'max_P': int(P.max()),
        'mean_layers': float(Ls.mean()), 'shape_groups': len(groups),
        'one_launch_ms': ms_var, 'one_launch_points_per_s': len(reqs) / (ms_var / 1e3),
        'grouped_ms': ms_grouped, 'grouped_points_per_s': len(reqs) / (ms_grouped / 1e3),
        'per_solve_ms_extrapolated': ms_single, 'per_solve_points_per_s': len(reqs) / (ms_single / 1e3),
        'orders_layers_per_s': float((P / 2 * Ls).sum() / (ms_var / 1e3)),
    }))


if __name__ == '__main__':
    main()
