"""Time the overlap integrals J and J_dag at a given size (FP64 GEMM path and
tensor-core split-TF32 path) on synthetic fields.

    python -m emustack_b200.profile_overlap [--cells N] [--nval M] [--max-order O]
                                            [--precision fp64|tf32x3|both] [--steps K] [--c64]

A square unit cell of N x N squares (2 N^2 P2 triangles), M Bloch modes with
random complex fields (reference layout [nel][M][13][3]) and the plane-wave
set of max order O at period 700 nm (--c64: the fields held as complex64,
tensor-core path only).  Prints one JSON line per precision with
the time per (J + J_dag) pair and the achieved rate against the algorithmic
count 2 * 8 * Npw * 2M * 6 nel flops.
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
    ap.add_argument('--cells', type=int, default=100)
    ap.add_argument('--nval', type=int, default=400)
    ap.add_argument('--max-order', type=int, default=10)
    ap.add_argument('--precision', default='both')
    ap.add_argument('--steps', type=int, default=3)
    ap.add_argument('--chunk', type=int, default=0)
    ap.add_argument('--c64', action='store_true', help='complex64 fields (tensor-core path)')
    args = ap.parse_args()
    from emustack_b200.films import grating_orders
    from emustack_b200.mesh import square_cell
    from emustack_b200.overlap import DeviceMesh, overlap_batch
    mesh = square_cell(args.cells, radius=0.3)
    dm = DeviceMesh(mesh)
    px, py = grating_orders(args.max_order, 700.0, 700.0)
    npw, M, nel = len(px), args.nval, mesh.nel
    g = torch.Generator(device='cuda').manual_seed(0)
    shape = (1, nel, M, 13, 3)
    s1 = torch.complex(torch.randn(shape, dtype=torch.float64, device='cuda', generator=g),
                       torch.randn(shape, dtype=torch.float64, device='cuda', generator=g))
    s2 = torch.complex(torch.randn(shape, dtype=torch.float64, device='cuda', generator=g),
                       torch.randn(shape, dtype=torch.float64, device='cuda', generator=g))
    if args.c64:
        s1, s2 = s1.to(torch.complex64), s2.to(torch.complex64)
    bloch = torch.tensor([[1e-6, 2e-7]], dtype=torch.float64, device='cuda')
    k0 = torch.tensor([2 * np.pi / (800.0 / 700.0)], dtype=torch.float64, device='cuda')
    flops = 2 * 8.0 * npw * 2 * M * 6 * nel
    precs = ['fp64', 'tf32x3'] if args.precision == 'both' else [args.precision]
    if args.c64:
        precs = ['tf32x3']
    for prec in precs:
        overlap_batch(dm, px, py, args.max_order, bloch, k0, s1, s2, precision=prec,
                      elements_per_chunk=args.chunk)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            overlap_batch(dm, px, py, args.max_order, bloch, k0, s1, s2, precision=prec,
                          elements_per_chunk=args.chunk)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        from emustack_b200.autotune import default_tuner
        tuned = [e['choice'] for k, e in default_tuner().log if '|overlap_tc|' in k]
        print(json.dumps({'precision': prec, 'fields': str(s1.dtype).replace('torch.', ''), 'nel': nel, 'nval': M, 'npw': npw, 'ms_per_J_pair': ms,
                          'tflops': flops / (ms / 1e3) / 1e12, 'flops': flops,
                          'tuned_chunk_splits': tuned[-1] if tuned else None}))


if __name__ == '__main__':
    main()
