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

With --arrays N, N array stacks (``array_stacks``) are solved, interfaces
included, three ways: grouped by shape on --streams streams (one
``emu_stack_dense_batch`` per group), as uneven batches of --array-chunk
stacks of any shapes in one ``emu_stack_var_batch`` launch each, and one
call per stack on a sample.
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


def prepare_array_groups(stacks, period=500.0, group=True):
    """Device inputs of the array stacks grouped by shape (P, number of
    layers), or one group per stack: air and substrate k_z, random J, J_dag,
    Bloch k_z, heights."""
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
    return prepared


def _group_layers(lay, n_air):
    """Interfaces of one group: film substrate, K array layers, air."""
    from emustack_b200.dense import DenseLayer, film_interface, interface_dense
    na, ns = n_air[lay['B']]
    Rs, Ts = film_interface(lay['kza'], na, lay['kzs'], ns, lay['wln'])
    Ra, Ta = film_interface(lay['kza'], na, lay['kza'], na, lay['wln'])
    layers = [DenseLayer(Rs, Ts, -Rs, Ts, False)]
    for k in range(lay['K']):
        R12, T12, R21, T21, _ = interface_dense(lay['kza'], na, lay['wln'], lay['J'][k], lay['Jd'][k])
        layers.append(DenseLayer(R12, T12, R21, T21, True, lay['kz'][k], lay['h'][k]))
    layers.append(DenseLayer(Ra, Ta, -Ra, Ta, False))
    return layers


def _n_air(prepared):
    dev = torch.device('cuda')
    return {B: (torch.ones(B, dtype=torch.complex128, device=dev),
                torch.full((B,), 1.46 + 0j, dtype=torch.complex128, device=dev))
            for B in sorted({lay['B'] for lay in prepared})}


def time_array_groups(stacks, period=500.0, group=True, n_streams=1):
    """Solve array stacks (interfaces + cascade + fluxes) grouped by shape
    (P, number of layers) into batched calls, or one call per stack; groups
    are dealt round-robin to n_streams CUDA streams (independent solves
    overlap on the device).  Returns (ms, groups).  Inputs are built on the
    device before timing."""
    from emustack_b200.dense import DenseStackSolver
    dev = torch.device('cuda')
    prepared = prepare_array_groups(stacks, period, group)
    streams = [torch.cuda.Stream(dev) for _ in range(n_streams)]
    solvers = [DenseStackSolver(dev) for _ in range(n_streams)]
    n_air = _n_air(prepared)

    def run(lay, solver):
        return solver.solve(_group_layers(lay, n_air), lay['P'], pol='TE', specular=lay['spec'],
                            num_prop=lay['nprop'])

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


def time_array_uneven(stacks, period=500.0, chunk=256, ws_budget_gb=40.0):
    """Solve the same array stacks with their interfaces computed per shape
    group and the cascades of up to `chunk` stacks of any shapes in ONE
    launch of the uneven dense batch (emu_stack_var_batch, one CTA per
    stack, costliest first).  Returns (ms, launches, slots)."""
    from emustack_b200.dense import StackVarSolver, VarStack
    dev = torch.device('cuda')
    prepared = prepare_array_groups(stacks, period, True)
    n_air = _n_air(prepared)
    solver = StackVarSolver(dev)
    # chunks of whole groups
    chunks, cur, n = [], [], 0
    for lay in prepared:
        cur.append(lay)
        n += lay['B']
        if n >= chunk:
            chunks.append(cur)
            cur, n = [], 0
    if cur:
        chunks.append(cur)

    def run(groups):
        vs, spec, nprop = [], [], []
        for lay in groups:
            layers = _group_layers(lay, n_air)
            for b in range(lay['B']):
                ls = []
                for j, dl in enumerate(layers):
                    kz = dl.kz[b] if dl.kz is not None else None
                    ls.append((dl.R12[b], dl.T12[b], dl.R21[b], dl.T21[b], dl.dense, kz, dl.height_norm))
                vs.append(VarStack(ls, lay['P'], pol='TE'))
            spec.append(lay['spec'])
            nprop.append(lay['nprop'])
        out = solver.solve(vs, spec=torch.cat(spec), num_prop=torch.cat(nprop),
                           ws_budget_bytes=ws_budget_gb * 1e9)
        # the chunk's interfaces and outputs are released here: the next
        # chunk's allocations on this stream are ordered after this launch
        return out['n_slots']

    run(chunks[0][:1])
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    slots = 0
    for c in chunks:
        slots = run(c)
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b), len(chunks), slots


def time_array_hybrid(stacks, period=500.0, d_split=256, chunk=1024, n_streams=4, ws_budget_gb=24.0):
    """Stacks with D = max(P, M) <= d_split as uneven one-launch batches on
    one stream, the larger ones grouped by shape (multi-CTA solves) on the
    other n_streams - 1 streams, all at once: the one-CTA-per-stack kernel
    fills the SMs the latency-bound multi-CTA steps leave idle.  Returns
    (ms, small stacks, large stacks)."""
    from emustack_b200.dense import DenseStackSolver, StackVarSolver, VarStack
    dev = torch.device('cuda')
    small = [s for s in stacks if 2 * s['npw'] + 20 <= d_split]
    large = [s for s in stacks if 2 * s['npw'] + 20 > d_split]
    prep_s = prepare_array_groups(small, period, True) if small else []
    prep_l = prepare_array_groups(large, period, True) if large else []
    n_air = _n_air(prep_s + prep_l)
    streams = [torch.cuda.Stream(dev) for _ in range(n_streams)]
    solvers = [DenseStackSolver(dev) for _ in range(n_streams)]
    var = StackVarSolver(dev)
    chunks, cur, n = [], [], 0
    for lay in prep_s:
        cur.append(lay)
        n += lay['B']
        if n >= chunk:
            chunks.append(cur)
            cur, n = [], 0
    if cur:
        chunks.append(cur)

    def run_small(groups):
        vs, spec, nprop = [], [], []
        for lay in groups:
            layers = _group_layers(lay, n_air)
            for b in range(lay['B']):
                vs.append(VarStack([(dl.R12[b], dl.T12[b], dl.R21[b], dl.T21[b], dl.dense,
                                     dl.kz[b] if dl.kz is not None else None, dl.height_norm)
                                    for dl in layers], lay['P'], pol='TE'))
            spec.append(lay['spec'])
            nprop.append(lay['nprop'])
        var.solve(vs, spec=torch.cat(spec), num_prop=torch.cat(nprop), ws_budget_bytes=ws_budget_gb * 1e9)

    def run_large(lay, solver):
        solver.solve(_group_layers(lay, n_air), lay['P'], pol='TE', specular=lay['spec'],
                     num_prop=lay['nprop'])

    if chunks:
        with torch.cuda.stream(streams[0]):
            run_small(chunks[0][:1])
    for lay in prep_l[:2]:
        run_large(lay, solvers[1])
    torch.cuda.synchronize()
    main_s = torch.cuda.current_stream(dev)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(main_s)
    for st in streams:
        st.wait_stream(main_s)
    with torch.cuda.stream(streams[0]):
        for c in chunks:
            run_small(c)
    for i, lay in enumerate(prep_l):
        k = 1 + i % (n_streams - 1)
        with torch.cuda.stream(streams[k]):
            run_large(lay, solvers[k])
    for st in streams:
        main_s.wait_stream(st)
    b.record(main_s)
    torch.cuda.synchronize()
    return a.elapsed_time(b), len(small), len(large)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--points', type=int, default=4096)
    ap.add_argument('--steps', type=int, default=5)
    ap.add_argument('--per-solve', type=int, default=512, help='points timed one launch each')
    ap.add_argument('--arrays', type=int, default=0, help='also time this many array stacks')
    ap.add_argument('--array-sample', type=int, default=32, help='array stacks timed one call each')
    ap.add_argument('--streams', type=int, default=4, help='streams for the array groups')
    ap.add_argument('--array-chunk', type=int, default=256, help='array stacks per uneven launch')
    ap.add_argument('--arrays-only', action='store_true', help='skip the film half')
    args = ap.parse_args()
    if args.arrays:
        stacks = array_stacks(args.arrays)
        ms_g, ng = time_array_groups(stacks, n_streams=args.streams)
        ms_h, n_small, n_large = time_array_hybrid(stacks, n_streams=args.streams)
        ms_u, n_launch, slots = time_array_uneven(stacks, chunk=args.array_chunk)
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
            'hybrid_ms': ms_h, 'hybrid_small_uneven': n_small, 'hybrid_large_grouped': n_large,
            'hybrid_solves_per_s': len(stacks) / (ms_h / 1e3), 'hybrid_tflops': flops / (ms_h / 1e3) / 1e12,
            'uneven_ms': ms_u, 'uneven_launches': n_launch, 'uneven_slots': slots,
            'uneven_solves_per_s': len(stacks) / (ms_u / 1e3), 'uneven_tflops': flops / (ms_u / 1e3) / 1e12,
            'per_solve_sample': len(sample), 'per_solve_ms_sample': ms_s,
            'per_solve_solves_per_s': len(sample) / (ms_s / 1e3),
        }), flush=True)
        if args.arrays_only:
            return
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
