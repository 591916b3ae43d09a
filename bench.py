"""Benchmark of the B200 GSM stage on the batched thin-film workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one batch): 10 films per stack (heights U(20,300) nm,
n U(1.3,4.0) + i U(0,0.5)) on an n=1.46 substrate under n=1.0, period
500 nm, max_order_PWs 5 (81 orders per polarisation, P = 162), evaluated at
2048 wavelengths U(350,1100) nm x 16 angles theta U(0,60), phi U(0,90)
(32768 spectral points), TE incidence, seeded synthetic data.  The metric is
R/T/A spectral points per second.

Arms
  ours       : device-resident inputs, one fused launch per step (`value`);
               `e2e` repeats the step through the public host-to-host API
               (FilmHostPipeline) with pinned host inputs: host->device
               copies, the solves and the device->host read of R_net/T_net
               diagonals and a/t/r lists, in 4096-point pieces on four
               streams so copies overlap solves.
  reference  : the reference's FP64 algorithm (the CPU oracle, a numpy
               restatement of backend/stack.py + backend/mode_calcs.py) on the
               host cores, a bounded sample per step.

Multi-GPU (torchrun): replicas; every rank solves its own full batch, no
collective on the data path (weak scaling); the step time is the max over
ranks.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_WL, N_ANG, N_FILMS = 2048, 16, 10
E2E_CHUNK, E2E_STREAMS = 4096, 4   # pieces of the host-to-host pipeline and their streams
PERIOD, MAX_ORDER, POL = 500.0, 5, 'TE'
METRIC = 'R/T/A spectral points/s (batched thin-film GSM, FP64)'
L2_FLUSH_BYTES = 256 << 20


def workload(seed=0):
    """Seeded synthetic inputs of the batched thin-film workload."""
    rng = np.random.default_rng(seed)
    h = rng.uniform(20, 300, N_FILMS)
    n = rng.uniform(1.3, 4.0, N_FILMS) + 1j * rng.uniform(0, 0.5, N_FILMS)
    n_stack = np.concatenate([[1.46 + 0j], n, [1.0 + 0j]])
    wl = rng.uniform(350, 1100, N_WL)
    th = rng.uniform(0, 60, N_ANG)
    ph = rng.uniform(0, 90, N_ANG)
    WL = np.repeat(wl, N_ANG)
    TH = np.tile(th, N_WL)
    PH = np.tile(ph, N_WL)
    # Light(wl, theta, phi): 1e-5 degree nudge and k_parallel (objects.py:1729-1743)
    THn = np.where(np.abs(TH) < 1e-5, TH + 1e-5, TH)
    PHn = np.where(np.abs(PH) < 1e-5, PH + 1e-5, PH)
    k = 2 * np.pi * 1.0 / WL
    t = THn * np.pi / 180
    p = PHn * np.pi / 180
    kp = np.stack([k * np.sin(t) * np.cos(p), k * np.sin(t) * np.sin(p)], axis=1)
    N = np.tile(n_stack, (WL.shape[0], 1))
    return dict(wl=WL, k_pll=np.ascontiguousarray(kp), n=N, heights=h, n_stack=n_stack,
                theta=TH, phi=PH)


CONFIG = {
    'workload': 'batched thin-film stacks: 10 films (h U(20,300) nm, n U(1.3,4.0)+iU(0,0.5)) '
                'on n=1.46 under n=1.0, period 500 nm, max_order_PWs=5 (81 orders/pol, P=162), '
                '2048 wavelengths U(350,1100) nm x 16 angles theta U(0,60), phi U(0,90), TE',
    'points_per_step': N_WL * N_ANG,
    'layers': N_FILMS + 2,
    'plane_waves': 162,
    'l2': 'flushed between timed steps (256 MiB write, untimed)',
}


# ---------------------------------------------------------------- oracle
def _oracle_point(args):
    os.environ.setdefault('OPENBLAS_NUM_THREADS', '1')
    from oracle import gsm_oracle as O
    n_stack, h, wl, kp = args
    r = O.film_stack_point(n_stack, h, wl, kp, PERIOD, max_order=MAX_ORDER, pol=POL)
    return float(r.a_list[-1]), float(r.r_list[0]), float(r.t_list[-1])


def cpu_reference(sample_points, seed=0, procs=None):
    """Time the reference algorithm (CPU oracle) on `sample_points` points,
    one single-threaded process per host core (as the reference's
    multiprocessing.Pool runs do, BLAS pinned to 1 thread)."""
    os.environ['OPENBLAS_NUM_THREADS'] = '1'
    os.environ['OMP_NUM_THREADS'] = '1'
    os.environ['MKL_NUM_THREADS'] = '1'
    w = workload(seed)
    rng = np.random.default_rng(seed + 1)
    idx = rng.choice(len(w['wl']), size=sample_points, replace=False)
    jobs = [(w['n_stack'], w['heights'], float(w['wl'][i]), w['k_pll'][i]) for i in idx]
    procs = procs or min(len(os.sched_getaffinity(0)), sample_points)
    ctx = mp.get_context('spawn')
    with ctx.Pool(procs) as pool:
        pool.map(_oracle_point, jobs[:procs])  # warm the workers (imports)
        t0 = time.perf_counter()
        pool.map(_oracle_point, jobs, chunksize=1)
        dt = time.perf_counter() - t0
    return sample_points / dt, procs, dt


# ---------------------------------------------------------------- clocks
class ClockSampler(object):
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
         'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
         'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', '-i', str(self.index), '--query-gpu=' + self.Q,
                 '--format=csv,noheader,nounits', '-lms', '100'],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ''
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for l in getattr(self, 'lines', []):
            f = [x.strip() for x in l.split(',')]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == 'active':
                    reasons.add(nm)
        if not sm:
            return {'sm_mhz': None, 'sm_max_mhz': mx, 'reasons': ['unsampled']}
        return {'sm_mhz': float(np.median(sm)), 'sm_max_mhz': mx, 'reasons': sorted(reasons),
                'samples': len(sm)}


# ---------------------------------------------------------------- GPU arm
def algorithmic_counts(B, L, P):
    """Algorithmic bytes of one batch: inputs read once (wl, k_pll, n) and the
    outputs written once (R_net, T_net diagonals, a/t lists, r, flags)."""
    by = B * (8 + 16 + 16 * L + 2 * 16 * P + 2 * 8 * (L - 1) + 8 + 4)
    return by


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from emustack_b200 import _lib
    from emustack_b200.films import FilmStackSolver
    from emustack_b200.probe import fp64_peak_tflops

    dev = torch.device('cuda', local_rank)
    torch.cuda.set_device(dev)
    lib = _lib.lib()
    w = workload(seed=0)
    B = len(w['wl'])
    L = N_FILMS + 2
    solver = FilmStackSolver(L, MAX_ORDER, PERIOD)
    P = solver.P
    d_wl = torch.tensor(w['wl'], device=dev)
    d_kp = torch.tensor(w['k_pll'], device=dev)
    d_n = torch.tensor(w['n'], device=dev)
    d_h = torch.tensor(w['heights'], device=dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()

    def step():
        return solver.solve(d_wl, d_kp, d_n, d_h, pol=POL)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    launches0 = lib.emu_launch_count()
    with ClockSampler(local_rank) as clk:
        for i in range(args.steps):
            flush.fill_(i & 0xff)
            starts[i].record(stream)
            step()
            ends[i].record(stream)
        torch.cuda.synchronize()
    launches = lib.emu_launch_count() - launches0
    if world > 1:
        dist.barrier()
    step_ms = np.array([s.elapsed_time(e) for s, e in zip(starts, ends)])
    tot = torch.tensor([step_ms.sum()], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(tot, op=dist.ReduceOp.MAX)
    total_ms = float(tot.item())
    ms_per_step = total_ms / args.steps
    value = world * B * args.steps / (total_ms / 1e3)

    # ---- e2e through the public host-to-host API (FilmHostPipeline): pinned
    # host inputs, the copies in, the solves and the copies out of R_net /
    # T_net diagonals and a/t/r lists, in pieces whose copies overlap the
    # solves of their neighbours
    from emustack_b200.films import FilmHostPipeline
    pipe = FilmHostPipeline(N_FILMS + 2, MAX_ORDER, PERIOD, device=dev, chunk=E2E_CHUNK, n_streams=E2E_STREAMS)
    h_wl = torch.from_numpy(w['wl']).pin_memory()
    h_kp = torch.from_numpy(w['k_pll']).pin_memory()
    h_n = torch.from_numpy(w['n']).pin_memory()
    h_h = torch.from_numpy(w['heights']).pin_memory()
    outs_h = pipe.outputs(B)
    h2d = sum(t.numel() * t.element_size() for t in (h_wl, h_kp, h_n, h_h))
    h2d += (h_h.numel() * h_h.element_size()) * ((B + E2E_CHUNK - 1) // E2E_CHUNK - 1)
    d2h = sum(t.numel() * t.element_size() for t in outs_h.values())

    def e2e_step():
        pipe.solve(h_wl, h_kp, h_n, h_h, pol=POL)

    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e_s = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e_e = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for i in range(args.steps):
        flush.fill_(i & 0xff)
        e_s[i].record(stream)
        e2e_step()
        e_e[i].record(stream)
    torch.cuda.synchronize()
    e_ms = np.array([s.elapsed_time(e) for s, e in zip(e_s, e_e)])
    etot = torch.tensor([e_ms.sum()], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(etot, op=dist.ReduceOp.MAX)
    e2e_value = world * B * args.steps / (float(etot.item()) / 1e3)
    # sanity: the copied results are the device results
    assert np.isfinite(outs_h['a_list'].numpy()).all()

    result = None
    if rank == 0:
        hbm = None
        try:
            with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
                peaks = json.load(f)
            hbm, hbm_src = float(peaks['hbm_gbs']), 'measured'
        except Exception:
            hbm, hbm_src = 6650.0, 'fallback'
        by = algorithmic_counts(B, L, P)
        achieved = by / (ms_per_step / 1e3) / 1e9
        flops = film_flops(B, L, P)
        fp64_peak = fp64_peak_tflops()
        tfl = flops / (ms_per_step / 1e3) / 1e12
        result = {
            'metric': METRIC,
            'value': value,
            'unit': 'points/s',
            'n_gpus': world,
            'steps': args.steps,
            'warmup': args.warmup,
            'ms_per_step': ms_per_step,
            'higher_is_better': True,
            'scaling': 'weak',
            'vs_baseline': None,
            'dtype': 'f64',
            'data': 'synthetic (seeded)',
            'config': dict(CONFIG, parallelism='replicas x%d' % world),
            'latency_ms': {'p50': float(np.percentile(step_ms, 50)),
                           'p99': float(np.percentile(step_ms, 99)),
                           'unit': 'one 32768-point batch'},
            'e2e': {'value': e2e_value, 'unit': 'points/s', 'h2d_bytes_per_step': h2d,
                    'd2h_bytes_per_step': d2h},
            'gpu_launches': int(launches),
            'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': hbm,
                         'unit': 'GB/s', 'frac': achieved / hbm, 'traffic': None,
                         'peak_source': hbm_src + ' (MEASURED_PEAKS.json hbm_gbs)',
                         'note': 'the kernel is FP64-issue bound, see compute'},
            'compute': {'bound': 'fp64', 'achieved_tflops': tfl, 'peak_tflops': fp64_peak,
                        'frac': tfl / fp64_peak if fp64_peak else None,
                        'peak_source': 'DFMA probe kernel (emu_probe_fp64), measured in this run',
                        'flops_per_step': flops,
                        'note': 'algorithmic flops count a divide, square root or exp as one'},
            'clocks': clk.summary(),
            'autotune': _tuned(),
        }
    return result


def _tuned():
    """Launch choices the autotuner made for the kernels timed here (chosen
    during warm-up from CUDA-event timings of every candidate)."""
    from emustack_b200.autotune import default_tuner
    return [{'kernel': k.split('|')[1], 'shape': json.loads(k.split('|')[2]), 'choice': e['choice'],
             'candidate_ms': {c: round(t, 4) for c, t in e['ms'].items()}}
            for k, e in default_tuner().log]


def film_flops(B, L, P):
    """Algorithmic FP64 operations of one batch of all-film stacks (each of
    + - * / sqrt counted as one): per (point, order, layer) the k_z square
    root argument and root (12), k and impedances (24), per polarisation the
    Fresnel pair (2 roots, 2 quotients: 40) and one cascade step (2 complex
    quotients, 6 complex products, 3 complex sums: 64)."""
    npw = P // 2
    per_order_layer = 12 + 24 + 2 * (40 + 64)
    return float(B) * npw * L * per_order_layer


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--cpu-sample', type=int, default=0,
                    help='points in the CPU sample (default: 8 per host core, >= 64)')
    args = ap.parse_args()
    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    local_rank = int(os.environ.get('LOCAL_RANK', '0'))
    cores = len(os.sched_getaffinity(0))
    sample = args.cpu_sample or max(64, 8 * cores)

    if args.impl == 'reference':
        if rank != 0:
            return
        vals = []
        for _ in range(max(1, args.steps)):
            v, procs, dt = cpu_reference(sample)
            vals.append(v)
        val = float(np.median(vals))
        line = {
            'impl': 'reference', 'metric': METRIC, 'value': val, 'unit': 'points/s',
            'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': 1e3 * sample / val, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic (seeded)',
            'config': dict(CONFIG, parallelism='host cores x%d' % procs),
            'cpu_baseline': {'value': val, 'unit': 'points/s', 'cores': procs, 'kind': 'port',
                             'sample': '%d random points of the batch per step, dense FP64 numpy '
                                       '(the reference algorithm), one process per core' % sample},
            'e2e': {'value': val, 'unit': 'points/s', 'h2d_bytes_per_step': 0,
                    'd2h_bytes_per_step': 0},
        }
        print(json.dumps(line))
        return

    # CPU baseline first, in spawned workers, before any GPU work
    cpu = None
    if rank == 0 and world == 1:
        v, procs, dt = cpu_reference(sample)
        cpu = {'value': v, 'unit': 'points/s', 'cores': procs, 'kind': 'port',
               'sample': '%d random points of the batch, dense FP64 numpy restatement of the '
                         'reference (oracle/gsm_oracle.py), one single-threaded process per core, '
                         '%.1f s' % (sample, dt)}
    import torch
    import torch.distributed as dist
    if world > 1:
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
    res = run_ours(args, rank, world, local_rank)
    if rank == 0:
        res['cpu_baseline'] = cpu
        print(json.dumps(res))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
