"""Time the whole per-wavelength GSM of the plain one-layer configuration,
eager and replayed from a CUDA graph.

    python -m emustack_b200.profile_config1 [--batch 50] [--cells 32] [--nval 60]
                                            [--max-order 3] [--precision fp64|tf32x3]

Stack: substrate n = 1.46 / one 2D square array, period 600 nm, cylinder
diameter 240 nm (mesh region of type 2), height 100 nm / air; max order 3
(Npw = 29, P = 58); `nval` Bloch modes with synthetic complex128 N(0,1)
fields per element node on a structured P2 mesh of 2 cells^2 triangles
(2 048 for 32 cells), propagation constants Re U(0, 2 k0), Im U(0, 0.1 k0);
`batch` wavelengths uniform in 400-900 nm at normal incidence (theta = phi
= 1e-5 deg as Light nudges them), TE.  One JSON line: ms per batch and
wavelengths/s for the eager chain and for the graph replay (inputs already
on the device; CUDA events).
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np
import torch

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--batch', type=int, default=50)
    ap.add_argument('--cells', type=int, default=32)
    ap.add_argument('--nval', type=int, default=60)
    ap.add_argument('--max-order', type=int, default=3)
    ap.add_argument('--precision', default='fp64')
    ap.add_argument('--steps', type=int, default=20)
    args = ap.parse_args()
    from emustack_b200.mesh import square_cell
    from emustack_b200.pipeline import NanoStackPipeline
    period, B, M = 600.0, args.batch, args.nval
    mesh = square_cell(args.cells, radius=120.0 / period)
    rng = np.random.default_rng(0)
    dev = torch.device('cuda')
    wl = np.linspace(400.0, 900.0, B)
    th = ph = np.radians(1e-5)
    k = 2 * np.pi / wl
    kp = np.stack([k * np.sin(th) * np.cos(ph), k * np.sin(th) * np.sin(ph)], axis=1)
    g = torch.Generator(device='cuda').manual_seed(0)
    shape = (B, mesh.nel, M, 13, 3)
    cr = lambda: torch.complex(torch.randn(shape, dtype=torch.float64, device=dev, generator=g),
                               torch.randn(shape, dtype=torch.float64, device=dev, generator=g))
    s1, s2 = cr(), cr()
    k0 = 2 * np.pi / (wl / period)
    beta = rng.uniform(0, 2, (B, M)) * k0[:, None] + 1j * rng.uniform(0, 0.1, (B, M)) * k0[:, None]
    pl = NanoStackPipeline(mesh, period, args.max_order, M, B, 100.0, precision=args.precision)
    pl.load(wl, kp, s1, s2, torch.tensor(beta, device=dev))
    del s1, s2
    ev = lambda: torch.cuda.Event(enable_timing=True)
    for _ in range(2):
        pl.forward()
    torch.cuda.synchronize()
    a, b = ev(), ev()
    a.record()
    for _ in range(args.steps):
        pl.forward()
    b.record()
    torch.cuda.synchronize()
    ms_eager = a.elapsed_time(b) / args.steps
    pl.capture()
    for _ in range(2):
        pl.replay()
    torch.cuda.synchronize()
    a.record()
    for _ in range(args.steps):
        pl.replay()
    b.record()
    torch.cuda.synchronize()
    ms_graph = a.elapsed_time(b) / args.steps
    nel, npw = mesh.nel, pl.npw
    P = 2 * npw
    flops_j = 2 * 8.0 * npw * 2 * M * 6 * nel
    flops_gsm = 8.0 * (3 * M * M * P + P * P * M + 4.0 / 3 * M ** 3) + \
        8.0 * (4.0 / 3 * P ** 3 + 5 * P * P * M + 3 * M * M * P + 4.0 / 3 * M ** 3)
    print(json.dumps({
        'batch': B, 'nel': nel, 'nval': M, 'npw': npw, 'precision': args.precision,
        'eager_ms_per_batch': ms_eager, 'graph_ms_per_batch': ms_graph,
        'eager_wl_per_s': B / (ms_eager / 1e3), 'graph_wl_per_s': B / (ms_graph / 1e3),
        'flops_per_wl': flops_j + flops_gsm,
        'graph_tflops': B * (flops_j + flops_gsm) / (ms_graph / 1e3) / 1e12,
    }))


if __name__ == '__main__':
    main()
