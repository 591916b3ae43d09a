"""Time an uneven batch of all-film solves in one launch against per-solve
and per-shape launches (and, with --arrays N, N nanostructured-array stacks
grouped by shape against one call per stack).

    python -m emustack_b200.profile_uneven [--points 4096] [--steps 5] [--arrays 2048]

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


def array_stacks(n, seed=0, period=500.0):
    """Nanostructured-array stacks of the uneven distribution: P = 2 Npw
    log-uniform in [50, 900] (nearest order set), M = P + 20 Bloch modes per
    array layer, 2-12 array layers between a film substrate (n = 1.46) and
    air.  Interfaces come from synthetic J (P x M), J_dag (M x P), complex
    N(0,1)/sqrt(P), Bloch k_z Re U(0, 2 k0), Im U(0, 0.1 k0), heights
    U(50, 200) nm; wavelength U(350, 1100) nm, normal incidence, TE."""
    from emustack_b200.serve_bench import order_table
    rng = np.random.default_rng(seed)
    tab = order_table(period)
    P = np.exp(rng.uniform(np.log(50), np.log(900), n))
    out = []
    for i in range(n):
        mo = int(np.argmin(np.abs(tab - P[i] / 2)))
        out.append(dict(mo=mo, npw=int(tab[mo]), K=int(rng.integers(2, 13)), wl=float(rng.uniform(350, 1100)),
                        seed=int(rng.integers(1 << 30))))
    return out


def time_array_groups(stacks, period=500.0, group=True, n_streams=1):
    """Solve array stacks (interfaces + cascade + fluxes) grouped by shape
    (P, number of layers) into batched calls, or one call per stack; groups
    are dealt round-robin to n_streams CUDA streams (independent solves
    overlap on the device).  Returns (ms, groups).  Inputs are built on the
    device before timing."""
    from emustack_b200.dense import DenseLayer, DenseStackSolver, film_interface, interface_dense
    from emustack_b200.films import grating_orders
    from emustack_b200.profile_dense import air_kz
    dev = torch.device('cuda')
    keyf = (lambda s: (s['mo'], s['K'])) if group else (lambda s: id(s))
    groups = collections.defaultdict(list)
    for s in stacks:
        groups[keyf(s)].append(s)
    prepared = []
    for _, ss in groups.items():
        mo, K = ss[0]['mo'], ss[0]['K']
        px, py = grating_orders(mo, period, period)
        npw = len(px)
        P, M, B = 2 * npw, 2 * npw + 20, len(ss)
        wl = np.array([s['wl'] for s in ss])
        wln = wl / period
        kza = np.stack([air_kz(px, py, w, period) for w in wl])
        order = np.argsort(-kza.real + kza.imag, axis=1, kind='stable')
        kza = np.take_along_axis(kza, order, 1)
        kzs = np.take_along_axis(np.stack([air_kz(px, py, w, period, 1.46) for w in wl]), order, 1)
        g = torch.Generator(device='cuda').manual_seed(ss[0]['seed'])
        cr = lambda *sh: torch.complex(torch.randn(sh, dtype=torch.float64, device=dev, generator=g),
                                       torch.randn(sh, dtype=torch.float64, device=dev, generator=g))
        k0 = torch.tensor(2 * np.pi / wln, device=dev)
        lay = dict(B=B, P=P, M=M, K=K, kza=torch.tensor(kza, device=dev), kzs=torch.tensor(kzs, device=dev),
                   wln=torch.tensor(wln, device=dev),
                   J=[cr(B, P, M) / np.sqrt(P) for _ in range(K)], Jd=[cr(B, M, P) / np.sqrt(P) for _ in range(K)],
                   kz=[torch.complex(2 * torch.rand(B, M, dtype=torch.float64, device=dev, generator=g),
                                     0.1 * torch.rand(B, M, dtype=torch.float64, device=dev, generator=g))
                       * k0[:, None] for _ in range(K)],
                   h=[float(x) for x in np.random.default_rng(ss[0]['seed']).uniform(50, 200, K) / period],
                   spec=torch.zeros(B, dtype=torch.int32, device=dev),
                   nprop=torch.tensor([[int((kza[b].imag == 0).sum())] * 2 + [int((kzs[b].imag == 0).sum())]
                                       for b in range(B)], dtype=torch.int32, device=dev))
        prepared.append(lay)
    streams = [torch.cuda.Stream(dev) for _ in range(n_streams)]
    solvers = [DenseStackSolver(dev) for _ in range(n_streams)]
    n_air = {}
    for B in sorted({lay['B'] for lay in prepared}):
        n_air[B] = (torch.ones(B, dtype=torch.complex128, device=dev),
                    torch.full((B,), 1.46 + 0j, dtype=torch.complex128, device=dev))

    def run(lay, solver):
        na, ns = n_air[lay['B']]
        Rs, Ts = film_interface(lay['kza'], na, lay['kzs'], ns, lay['wln'])
        Ra, Ta = film_interface(lay['kza'], na, lay['kza'], na, lay['wln'])
        layers = [DenseLayer(Rs, Ts, -Rs, Ts, False)]
        for k in range(lay['K']):
            R12, T12, R21, T21, _ = interface_dense(lay['kza'], na, lay['wln'], lay['J'][k], lay['Jd'][k])
            layers.append(DenseLayer(R12, T12, R21, T21, True, lay['kz'][k], lay['h'][k]))
        layers.append(DenseLayer(Ra, Ta, -Ra, Ta, False))
        return solver.solve(layers, lay['P'], pol='TE', specular=lay['spec'], num_prop=lay['nprop'])

    for lay in prepared[:3]:
        run(lay, solvers[0])
    torch.cuda.synchronize()
    main = torch.cuda.current_stream(dev)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(main)
    for st in streams:
        st.wait_stream(main)
    for i, lay in enumerate(prepared):
        with torch.cuda.stream(streams[i % n_streams]):
            run(lay, solvers[i % n_streams])
    for st in streams:
        main.wait_stream(st)
    b.record(main)
    torch.cuda.synchronize()
    return a.elapsed_time(b), len(prepared)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--points', type=int, default=4096)
    ap.add_argument('--steps', type=int, default=5)
    ap.add_argument('--per-solve', type=int, default=512, help='points timed one launch each')
    ap.add_argument('--arrays', type=int, default=0, help='also time this many array stacks')
    ap.add_argument('--array-sample', type=int, default=32, help='array stacks timed one call each')
    ap.add_argument('--streams', type=int, default=4, help='streams for the array groups')
    args = ap.parse_args()
    if args.arrays:
        stacks = array_stacks(args.arrays)
        ms_g, ng = time_array_groups(stacks, n_streams=args.streams)
        sample = stacks[:args.array_sample]
        ms_s, _ = time_array_groups(sample, group=False)
        flops = 0.0
        for s in stacks:
            P = 2 * s['npw']
            M = P + 20
            flops += s['K'] * 8.0 * ((3 * M * M * P + P * P * M + 4.0 / 3 * M ** 3)
                                     + (4.0 / 3 * P ** 3 + 5 * P * P * M + 3 * M * M * P + 4.0 / 3 * M ** 3))
        print(json.dumps({
            'array_stacks': len(stacks), 'shape_groups': ng, 'streams': args.streams,
            'mean_P': float(np.mean([2 * s['npw'] for s in stacks])),
            'mean_array_layers': float(np.mean([s['K'] for s in stacks])),
            'grouped_ms': ms_g, 'grouped_solves_per_s': len(stacks) / (ms_g / 1e3),
            'grouped_tflops': flops / (ms_g / 1e3) / 1e12,
            'per_solve_sample': len(sample), 'per_solve_ms_sample': ms_s,
            'per_solve_solves_per_s': len(sample) / (ms_s / 1e3),
        }), flush=True)
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
