"""Time the dense GSM stage (film/nanostructure interfaces + cascade + fluxes)
on synthetic layers of a given shape.

    python -m emustack_b200.profile_dense [--npw-order O] [--period D] [--nval M]
                                          [--layers K] [--batch B] [--steps S] [--mode 0|1|2]
    python -m emustack_b200.profile_dense --gemm [--batch B]   (the complex GEMM alone)

Substrate n=1.46 and superstrate air are films; K nanostructured layers of M
Bloch modes sit between them with random J (P x M) and J_dag (M x P), complex
N(0,1)/sqrt(P), random k_z (Re U(0, 2k0), Im U(0, 0.1 k0)) and heights
U(50, 200) nm.  B wavelengths U(400, 900) nm at normal incidence, TE.
Prints one JSON line: ms per wavelength for the K interfaces
(backend/mode_calcs.py:480-515) and for the cascade + fluxes
(backend/stack.py:196-426), with the algorithmic FP64 flop counts
  interface: 8 (3 M^2 P + P^2 M + 4/3 M^3)
  cascade:   8 (4/3 P^3 + 5 P^2 M + 3 M^2 P + 4/3 M^3) per finite layer
and the achieved rate against the measured FP64 FMA peak.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np
import torch

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def air_kz(px, py, wl, period, n=1.0):
    k = 2 * np.pi * n / (wl / period)
    al = 2 * np.pi * px + 2 * np.pi * 1e-12
    be = 2 * np.pi * py
    kz = np.sqrt((k * k - al * al - be * be).astype(np.complex128))
    return kz


def gemm_rate(args):
    """TFLOP/s of the batched complex GEMM C[P x M] = A[P x P] B[P x M] over
    the batch, 8 P^2 M real flop each."""
    from emustack_b200.dense import zgemm_batched
    from emustack_b200.films import grating_orders
    from emustack_b200.probe import fp64_peak_tflops
    dev = torch.device('cuda')
    P = 2 * len(grating_orders(args.max_order, args.period, args.period)[0])
    M, B = args.nval, args.batch
    g = torch.Generator(device='cuda').manual_seed(0)
    cr = lambda *sh: torch.complex(torch.randn(sh, dtype=torch.float64, device=dev, generator=g),
                                   torch.randn(sh, dtype=torch.float64, device=dev, generator=g))
    A, Bm = cr(B, P, P), cr(B, P, M)
    C_ = torch.empty(B, P, M, dtype=torch.complex128, device=dev)
    for _ in range(max(args.warmup, 1)):
        zgemm_batched(A, Bm, C_)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    torch.cuda.synchronize()
    ev[0].record()
    for _ in range(args.steps):
        zgemm_batched(A, Bm, C_)
    ev[1].record()
    torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[1]) / args.steps
    tf = B * 8.0 * P * P * M / (ms / 1e3) / 1e12
    peak = fp64_peak_tflops()
    print(json.dumps({'gemm': [P, P, M], 'batch': B, 'ms': ms, 'tflops': tf, 'fp64_peak_tflops': peak,
                      'frac': tf / peak}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--max-order', type=int, default=10)
    ap.add_argument('--period', type=float, default=700.0)
    ap.add_argument('--nval', type=int, default=400)
    ap.add_argument('--layers', type=int, default=4)
    ap.add_argument('--batch', type=int, default=148)
    ap.add_argument('--steps', type=int, default=2)
    ap.add_argument('--warmup', type=int, default=1)
    ap.add_argument('--mode', type=int, default=0, help='cascade: 0 auto, 1 one CTA per solve, 2 multi-CTA')
    ap.add_argument('--gemm', action='store_true',
                    help='time only the batched complex GEMM (emu_zgemm_batched) at P x P x M')
    args = ap.parse_args()
    if args.gemm:
        return gemm_rate(args)
    from emustack_b200.dense import DenseLayer, DenseStackSolver, film_interface, interface_dense
    from emustack_b200.films import grating_orders
    from emustack_b200.probe import fp64_peak_tflops
    dev = torch.device('cuda')
    rng = np.random.default_rng(0)
    px, py = grating_orders(args.max_order, args.period, args.period)
    npw = len(px)
    P, M, B, K = 2 * npw, args.nval, args.batch, args.layers
    wl = rng.uniform(400.0, 900.0, B)
    wln = wl / args.period
    kz_air = np.stack([air_kz(px, py, w, args.period) for w in wl])
    order = np.argsort(-kz_air.real + kz_air.imag, axis=1, kind='stable')
    kz_air = np.take_along_axis(kz_air, order, 1)
    kz_sub = np.stack([air_kz(px, py, w, args.period, 1.46) for w in wl])
    kz_sub = np.take_along_axis(kz_sub, order, 1)
    t = lambda a, dt=torch.complex128: torch.tensor(a, dtype=dt, device=dev)
    d_kair, d_ksub = t(kz_air), t(kz_sub)
    n_air = torch.ones(B, dtype=torch.complex128, device=dev)
    n_sub = torch.full((B,), 1.46 + 0j, dtype=torch.complex128, device=dev)
    d_wln = t(wln, torch.float64)
    g = torch.Generator(device='cuda').manual_seed(0)

    def crandn(*shape):
        return torch.complex(torch.randn(shape, dtype=torch.float64, device=dev, generator=g),
                             torch.randn(shape, dtype=torch.float64, device=dev, generator=g))

    Js = [crandn(B, P, M) / np.sqrt(P) for _ in range(K)]
    Jds = [crandn(B, M, P) / np.sqrt(P) for _ in range(K)]
    k0 = 2 * np.pi / wln
    kzs = []
    for _ in range(K):
        re = rng.uniform(0, 2, (B, M)) * k0[:, None]
        im = rng.uniform(0, 0.1, (B, M)) * k0[:, None]
        kzs.append(t(re + 1j * im))
    hs = rng.uniform(50.0, 200.0, K) / args.period

    def interfaces():
        out = []
        for k in range(K):
            out.append(interface_dense(d_kair, n_air, d_wln, Js[k], Jds[k]))
        return out

    def films():
        Rs, Ts = film_interface(d_kair, n_air, d_ksub, n_sub, d_wln)
        Ra, Ta = film_interface(d_kair, n_air, d_kair, n_air, d_wln)
        return (Rs, Ts), (Ra, Ta)

    solver = DenseStackSolver(dev)
    spec = torch.zeros(B, dtype=torch.int32, device=dev)
    nprop = torch.tensor([[int((kz_air[b].imag == 0).sum()), int((kz_air[b].imag == 0).sum()),
                           int((kz_sub[b].imag == 0).sum())] for b in range(B)],
                         dtype=torch.int32, device=dev)

    def cascade(ifs, fl):
        (Rs, Ts), (Ra, Ta) = fl
        lay = [DenseLayer(Rs, Ts, -Rs, Ts, False)]
        for k in range(K):
            R12, T12, R21, T21, _ = ifs[k]
            lay.append(DenseLayer(R12, T12, R21, T21, True, kzs[k], hs[k]))
        lay.append(DenseLayer(Ra, Ta, -Ra, Ta, False))
        return solver.solve(lay, P, pol='TE', specular=spec, num_prop=nprop, mode=args.mode)

    for _ in range(args.warmup):
        ifs = interfaces()
        cascade(ifs, films())
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    t_if = t_cs = 0.0
    for _ in range(args.steps):
        ev[0].record()
        ifs = interfaces()
        fl = films()
        ev[1].record()
        out = cascade(ifs, fl)
        ev[2].record()
        torch.cuda.synchronize()
        t_if += ev[0].elapsed_time(ev[1])
        t_cs += ev[1].elapsed_time(ev[2])
    t_if /= args.steps
    t_cs /= args.steps
    f_if = K * 8.0 * (3 * M * M * P + P * P * M + 4.0 / 3 * M ** 3)
    f_cs = K * 8.0 * (4.0 / 3 * P ** 3 + 5 * P * P * M + 3 * M * M * P + 4.0 / 3 * M ** 3)
    peak = fp64_peak_tflops()
    info = out['info'].cpu().numpy()
    rate = lambda f, ms: B * f / (ms / 1e3) / 1e12
    print(json.dumps({
        'P': P, 'M': M, 'layers': K, 'batch': B, 'mode': args.mode,
        'interfaces_ms_per_wl': t_if / B, 'cascade_ms_per_wl': t_cs / B,
        'total_ms_per_wl': (t_if + t_cs) / B, 'wl_per_s': B / ((t_if + t_cs) / 1e3),
        'interfaces_tflops': rate(f_if, t_if), 'cascade_tflops': rate(f_cs, t_cs),
        'fp64_peak_tflops': peak, 'interfaces_frac': rate(f_if, t_if) / peak,
        'cascade_frac': rate(f_cs, t_cs) / peak, 'singular': int((info != 0).sum()),
        'flops_per_wl': f_if + f_cs,
    }))


if __name__ == '__main__':
    main()
