"""Benchmark of the B200 GSM stage.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config 1|2|3|4|5] [--no-extras]

Headline workload (config 2, the default; one "step" = one batch): 10 films
per stack (heights U(20,300) nm, n U(1.3,4.0) + i U(0,0.5)) on an n=1.46
substrate under n=1.0, period 500 nm, max_order_PWs 5 (81 orders per
polarisation, P = 162), evaluated at 2048 wavelengths U(350,1100) nm x 16
angles theta U(0,60), phi U(0,90) (32768 spectral points), TE incidence,
seeded synthetic data.  The metric is R/T/A spectral points per second.

Arms
  ours       : device-resident inputs, one fused launch per step (`value`);
               `e2e` repeats the step through the public host-to-host API
               (FilmHostPipeline) with pinned host inputs: host->device
               copies, the solves and the device->host read of every
               point's R/T/A (a/t/r lists and flags), in 4096-point pieces
               on four streams so copies overlap solves;
               `e2e_with_R_T_net` also reads the R_net / T_net diagonals
               back (176 MB per step: the host link bounds it).  Unless --no-extras, the
               same JSON line carries `north_star`: the batched GSM against
               the plain FP64 GPU GSM (this library called once per solve,
               the way the reference calls its GSM) on config 2, on the
               config-1 chain (tensor-core J) and on a config-4 mix of
               uneven film and array solves, and a short Poisson-arrival
               serving run (config 5) with request p50 / p99 latency.
  reference  : the reference's FP64 algorithm (the CPU oracle, a numpy
               restatement of backend/stack.py + backend/mode_calcs.py) on the
               host cores, a bounded sample per step.

--config 1|3|4|5 prints one JSON line of that workload alone, in more depth
(the commands under profiles/ use them); --config 2 is the contract line.

Multi-GPU (torchrun): replicas; every rank solves its own full batch, no
collective on the data path (weak scaling); the step time is the max over
ranks.
"""
from __future__ import annotations

import argparse
import collections
import gc
import itertools
import json
import multiprocessing as mp
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_WL, N_ANG, N_FILMS = 2048, 16, 10
E2E_CHUNK, E2E_STREAMS = 4096, 4   # pieces of the host-to-host pipeline and their streams
PERIOD, MAX_ORDER, POL = 500.0, 5, 'TE'
METRIC = 'R/T/A spectral points/s (batched thin-film GSM, FP64)'
L2_FLUSH_BYTES = 256 << 20
# DRAM bytes of one 32768-point launch of the bench kernel, from one ncu
# capture (dram__bytes_read.sum + dram__bytes_write.sum); reported only when
# the autotuner picks the captured launch variant
NCU_TRAFFIC = {'bytes': 169334528, 'variant': 4, 'kernel': 'film_stack_kernel<256, 3, true>',
               'kernel_ms_under_ncu': 1.062,
               'source': 'ncu --set full capture, profiles/film_stack_32768pts.md'}


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


def _events(n):
    import torch
    return [torch.cuda.Event(enable_timing=True) for _ in range(n)]


def hbm_peak():
    """HBM copy bandwidth (GB/s) measured on this pool's B200s, else the
    earlier measurement used as the fallback."""
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            return float(json.load(f)['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


def _timed(fn, steps, warmup=2, flush=None):
    """Median ms of `steps` calls of fn (CUDA events on the current stream,
    after `warmup` untimed calls; L2 flushed before each timed call when a
    flush buffer is given)."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ts = []
    for i in range(steps):
        if flush is not None:
            flush.fill_(i & 0xff)
        a, b = _events(2)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    return float(np.median(ts))


# ---------------------------------------------------------------- config 2
def algorithmic_counts(B, L, P):
    """Algorithmic bytes of one batch: inputs read once (wl, k_pll, n) and the
    outputs written once (R_net, T_net diagonals, a/t lists, r, flags)."""
    by = B * (8 + 16 + 16 * L + 2 * 16 * P + 2 * 8 * (L - 1) + 8 + 4)
    return by


def film_flops(B, L, P):
    """Algorithmic FP64 operations of one batch of all-film stacks (each of
    + - * / sqrt counted as one), counted on the reference's recursion for
    diagonal matrices: per (point, order, layer) the k_z square root
    argument and root (12), k and impedances (24), per polarisation the
    Fresnel pair (2 roots, 2 quotients: 40) and one cascade step (2 complex
    quotients, 6 complex products, 3 complex sums: 64).  The kernel's
    one-quotient form does less arithmetic than this count."""
    npw = P // 2
    per_order_layer = 12 + 24 + 2 * (40 + 64)
    return float(B) * npw * L * per_order_layer


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
    starts = _events(args.steps)
    ends = _events(args.steps)
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
    h_wl = torch.from_numpy(w['wl']).pin_memory()
    h_kp = torch.from_numpy(w['k_pll']).pin_memory()
    h_n = torch.from_numpy(w['n']).pin_memory()
    h_h = torch.from_numpy(w['heights']).pin_memory()

    def e2e_run(outputs):
        """points/s through FilmHostPipeline bringing `outputs` back to the
        host, and the bytes copied each way per step"""
        pipe = FilmHostPipeline(N_FILMS + 2, MAX_ORDER, PERIOD, device=dev, chunk=E2E_CHUNK,
                                n_streams=E2E_STREAMS, outputs=outputs)
        outs_h = pipe.outputs(B)
        h2d = sum(t.numel() * t.element_size() for t in (h_wl, h_kp, h_n, h_h))
        h2d += (h_h.numel() * h_h.element_size()) * ((B + E2E_CHUNK - 1) // E2E_CHUNK - 1)
        d2h = sum(t.numel() * t.element_size() for t in outs_h.values())
        for _ in range(args.warmup):
            pipe.solve(h_wl, h_kp, h_n, h_h, pol=POL)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e_s, e_e = _events(args.steps), _events(args.steps)
        for i in range(args.steps):
            flush.fill_(i & 0xff)
            e_s[i].record(stream)
            pipe.solve(h_wl, h_kp, h_n, h_h, pol=POL)
            e_e[i].record(stream)
        torch.cuda.synchronize()
        e_ms = np.array([s.elapsed_time(e) for s, e in zip(e_s, e_e)])
        etot = torch.tensor([e_ms.sum()], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(etot, op=dist.ReduceOp.MAX)
        # sanity: the copied results are the device results' lists
        assert np.isfinite(outs_h['a_list'].numpy()).all()
        return world * B * args.steps / (float(etot.item()) / 1e3), h2d, d2h

    # the metric's result per point is its R/T/A: the a/t/r lists come back;
    # the same with the R_net / T_net diagonals as well is reported beside it
    e2e_value, h2d, d2h = e2e_run(FilmHostPipeline.SPECTRA)
    e2e_full, h2d_f, d2h_f = e2e_run(FilmHostPipeline.OUT)

    result = None
    if rank == 0:
        hbm, hbm_src = hbm_peak()
        by = algorithmic_counts(B, L, P)
        achieved = by / (ms_per_step / 1e3) / 1e9
        flops = film_flops(B, L, P)
        fp64_peak = fp64_peak_tflops()
        tuned = _tuned()
        variant = next((t['choice'] for t in tuned if t['kernel'] == 'film_stack' and
                        t['shape'].get('B') == _bucket(B) and not t['shape'].get('inc')), None)
        traffic = NCU_TRAFFIC['bytes'] if variant == NCU_TRAFFIC['variant'] else None
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
                    'd2h_bytes_per_step': d2h,
                    'result': 'a_list, t_list, r_list and flags of every point (the R/T/A spectra)'},
            'e2e_with_R_T_net': {'value': e2e_full, 'unit': 'points/s', 'h2d_bytes_per_step': h2d_f,
                                 'd2h_bytes_per_step': d2h_f,
                                 'result': 'the R/T/A spectra and the R_net / T_net diagonals'},
            'gpu_launches': int(launches),
            'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': hbm,
                         'unit': 'GB/s', 'frac': achieved / hbm, 'traffic': traffic,
                         'traffic_source': dict(NCU_TRAFFIC, launch_variant_now=variant),
                         'peak_source': hbm_src + ' (MEASURED_PEAKS.json hbm_gbs)',
                         'note': 'the kernel is FP64-issue bound, see compute'},
            'compute': {'bound': 'fp64', 'achieved_tflops': tfl, 'peak_tflops': fp64_peak,
                        'frac': tfl / fp64_peak if fp64_peak else None,
                        'peak_source': 'DFMA probe kernel (emu_probe_fp64), measured in this run',
                        'flops_per_step': flops,
                        'note': 'algorithmic flops count a divide, square root or exp as one'},
            'clocks': clk.summary(),
            'autotune': tuned,
        }
        if not args.no_extras:
            result['north_star'] = north_star_extras(dev, w, solver, value)
    return result


def _bucket(n):
    from emustack_b200.autotune import size_bucket
    return size_bucket(n)


def _tuned():
    """Launch choices the autotuner holds for the kernels timed here (chosen
    from CUDA-event timings of every candidate, in warm-up or read from its
    cache file)."""
    from emustack_b200.autotune import default_tuner
    out = []
    for k, e in default_tuner().cache.items():
        fam, shape = k.split('|')[1], json.loads(k.split('|')[2])
        if fam == 'film_stack' and shape.get('L') == N_FILMS + 2 and shape.get('npw') == len(order_table_npw()):
            out.append({'kernel': fam, 'shape': shape, 'choice': e['choice'],
                        'candidate_ms': {c: round(t, 4) for c, t in e['ms'].items()}})
    return out


def order_table_npw():
    """Orders per polarisation of the bench workload."""
    from emustack_b200.films import grating_orders
    return grating_orders(MAX_ORDER, PERIOD, PERIOD)[0]


# ---------------------------------------------------------------- extras
def plain_config2(dev, w, n_points=1024):
    """The plain FP64 GPU GSM on the config-2 points: one spectral point per
    call of the public solver (emu_film_stack_batch with B = 1), inputs
    already on the device, as the reference calls its GSM once per
    Stack.calc_scat.  Returns points/s."""
    import torch
    from emustack_b200.films import FilmStackSolver
    s = FilmStackSolver(N_FILMS + 2, MAX_ORDER, PERIOD, device=dev)
    idx = np.random.default_rng(5).choice(len(w['wl']), n_points, replace=False)
    pts = [(torch.tensor(w['wl'][i:i + 1], device=dev), torch.tensor(w['k_pll'][i:i + 1], device=dev),
            torch.tensor(w['n'][i:i + 1], device=dev)) for i in idx]
    h = torch.tensor(w['heights'], device=dev)

    def run():
        for wl, kp, n in pts:
            s.solve(wl, kp, n, h, pol=POL)

    ms = _timed(run, 3, warmup=1)
    return n_points / (ms / 1e3)


def order_table(period, max_mo=16):
    from emustack_b200.films import grating_orders
    return np.array([len(grating_orders(m, period, period)[0]) for m in range(max_mo + 1)])


def film_requests(n, seed=0, period=500.0):
    """Uneven all-film solves of the uneven-batch distribution: P = 2 Npw
    log-uniform in [50, 900] (the order set of the max order whose Npw is
    nearest), 2-12 finite layers, n U(1.3, 4.0) + i U(0, 0.5) on n = 1.46
    under air, heights U(20, 300) nm, wavelength U(350, 1100) nm, theta
    U(0, 60), phi U(0, 90) degrees, polarisations TE / TM / un / R Circ."""
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


def time_film_mix(dev, reqs, per_solve=256):
    """Uneven film solves: one emu_film_var_batch launch for all of them
    against one emu_film_stack_batch launch per solve (a sample,
    extrapolated).  Returns (batched ms, per-solve ms) for the whole set."""
    import torch
    from emustack_b200.films import FilmStackSolver, FilmVarSolver
    vs = FilmVarSolver(dev)
    pl = vs.plan(reqs)
    ms_var = _timed(lambda: vs.solve(pl), 5, warmup=2)
    single = []
    for r in reqs[:per_solve]:
        L = len(r.n)
        s = FilmStackSolver(L, r.max_order, 500.0, device=dev)
        single.append((s, torch.tensor([r.wl_nm], dtype=torch.float64, device=dev),
                       torch.tensor(r.k_pll.reshape(1, 2), dtype=torch.float64, device=dev),
                       torch.tensor(r.n.reshape(1, L), dtype=torch.complex128, device=dev),
                       torch.tensor(r.heights, dtype=torch.float64, device=dev), r.pol))

    def run():
        for s, wl, kp, n, h, pol in single:
            s.solve(wl, kp, n, h, pol=pol)

    ms_one = _timed(run, 2, warmup=1) / len(single) * len(reqs)
    return ms_var, ms_one


def array_stack_specs(n, seed=0, period=500.0):
    """Nanostructured-array stacks of the uneven distribution: P = 2 Npw
    log-uniform in [50, 900] (nearest order set), M = P + 20 Bloch modes per
    array layer (the reference's default num_BMs), 2-12 array layers between
    a film substrate (n = 1.46) and air, heights U(50, 200) nm, wavelength
    U(350, 1100) nm, normal incidence, TE.  The layers' J (P x M) and J_dag
    (M x P) are complex N(0,1)/sqrt(P), Bloch k_z Re U(0, 2 k0),
    Im U(0, 0.1 k0)."""
    rng = np.random.default_rng(seed)
    tab = order_table(period)
    P = np.exp(rng.uniform(np.log(50), np.log(900), n))
    out = []
    for i in range(n):
        mo = int(np.argmin(np.abs(tab - P[i] / 2)))
        out.append(dict(mo=mo, npw=int(tab[mo]), K=int(rng.integers(2, 13)), wl=float(rng.uniform(350, 1100)),
                        seed=int(rng.integers(1 << 30))))
    return out


def _air_kz(px, py, wl, period, n=1.0):
    k = 2 * np.pi * n / (wl / period)
    al = 2 * np.pi * px + 2 * np.pi * 1e-12
    be = 2 * np.pi * py
    return np.sqrt((k * k - al * al - be * be).astype(np.complex128))


def prepare_array_groups(stacks, period=500.0, group=True):
    """Device inputs of the array stacks grouped by shape (order set,
    number of layers), or one group per stack."""
    import torch
    from emustack_b200.films import grating_orders
    dev = torch.device('cuda')
    keyf = (lambda s: (s['mo'], s['K'], s.get('M'))) if group else (lambda s: id(s))
    groups = collections.defaultdict(list)
    for s in stacks:
        groups[keyf(s)].append(s)
    prepared = []
    for _, ss in groups.items():
        mo, K = ss[0]['mo'], ss[0]['K']
        px, py = grating_orders(mo, period, period)
        npw = len(px)
        P, B = 2 * npw, len(ss)
        M = ss[0].get('M') or P + 20    # Bloch modes per array layer (default: the reference's num_BMs)
        wl = np.array([s['wl'] for s in ss])
        wln = wl / period
        kza = np.stack([_air_kz(px, py, x, period) for x in wl])
        order = np.argsort(-kza.real + kza.imag, axis=1, kind='stable')
        kza = np.take_along_axis(kza, order, 1)
        kzs = np.take_along_axis(np.stack([_air_kz(px, py, x, period, 1.46) for x in wl]), order, 1)
        g = torch.Generator(device='cuda').manual_seed(ss[0]['seed'])
        cr = lambda *sh: torch.complex(torch.randn(sh, dtype=torch.float64, device=dev, generator=g),
                                       torch.randn(sh, dtype=torch.float64, device=dev, generator=g))
        k0 = torch.tensor(2 * np.pi / wln, device=dev)
        prepared.append(dict(
            B=B, P=P, M=M, K=K, kza=torch.tensor(kza, device=dev), kzs=torch.tensor(kzs, device=dev),
            wln=torch.tensor(wln, device=dev),
            J=[cr(B, P, M) / np.sqrt(P) for _ in range(K)], Jd=[cr(B, M, P) / np.sqrt(P) for _ in range(K)],
            kz=[torch.complex(2 * torch.rand(B, M, dtype=torch.float64, device=dev, generator=g),
                              0.1 * torch.rand(B, M, dtype=torch.float64, device=dev, generator=g))
                * k0[:, None] for _ in range(K)],
            h=[float(x) for x in np.random.default_rng(ss[0]['seed']).uniform(50, 200, K) / period],
            spec=torch.zeros(B, dtype=torch.int32, device=dev),
            nprop=torch.tensor([[int((kza[b].imag == 0).sum())] * 2 + [int((kzs[b].imag == 0).sum())]
                                for b in range(B)], dtype=torch.int32, device=dev)))
    return prepared


def _group_layers(lay):
    """Interfaces of one group (film substrate, K array layers, air)."""
    import torch
    from emustack_b200.dense import DenseLayer, film_interface, interface_dense
    B = lay['B']
    dev = lay['kza'].device
    na = torch.ones(B, dtype=torch.complex128, device=dev)
    ns = torch.full((B,), 1.46 + 0j, dtype=torch.complex128, device=dev)
    Rs, Ts = film_interface(lay['kza'], na, lay['kzs'], ns, lay['wln'])
    Ra, Ta = film_interface(lay['kza'], na, lay['kza'], na, lay['wln'])
    layers = [DenseLayer(Rs, Ts, -Rs, Ts, False)]
    for k in range(lay['K']):
        R12, T12, R21, T21, _ = interface_dense(lay['kza'], na, lay['wln'], lay['J'][k], lay['Jd'][k])
        layers.append(DenseLayer(R12, T12, R21, T21, True, lay['kz'][k], lay['h'][k]))
    layers.append(DenseLayer(Ra, Ta, -Ra, Ta, False))
    return layers


def time_array_stacks(stacks, group=True, n_streams=4):
    """Array stacks, interfaces included: grouped by shape into batched
    calls dealt round-robin to n_streams streams, or one call per stack.
    Returns ms for the set."""
    import torch
    from emustack_b200.dense import DenseStackSolver
    dev = torch.device('cuda')
    prepared = prepare_array_groups(stacks, group=group)
    streams = [torch.cuda.Stream(dev) for _ in range(n_streams)]
    solvers = [DenseStackSolver(dev) for _ in range(n_streams)]

    def one(lay, solver):
        solver.solve(_group_layers(lay), lay['P'], pol='TE', specular=lay['spec'], num_prop=lay['nprop'])

    def run():
        main = torch.cuda.current_stream(dev)
        for st in streams:
            st.wait_stream(main)
        for i, lay in enumerate(prepared):
            with torch.cuda.stream(streams[i % n_streams]):
                one(lay, solvers[i % n_streams])
        for st in streams:
            main.wait_stream(st)

    return _timed(run, 1, warmup=1)


def config1_chain(dev, batch=50, steps=10):
    """Config-1 chain (film k_z, adjoint normalisation, J / J_dag,
    interfaces, cascade, fluxes) of one 2D array (period 600 nm, 2048-
    triangle P2 mesh, 60 Bloch modes, max order 3) at `batch` wavelengths
    400-900 nm: plain = one wavelength per call, FP64 J, eager; batched =
    all wavelengths in one CUDA graph with the tensor-core (split-TF32 x3) J.
    Returns wavelengths/s of both and the largest |delta| of the a/t/r lists
    of the batched tensor-core chain against the batched FP64 chain."""
    import torch
    from emustack_b200.mesh import square_cell
    from emustack_b200.pipeline import NanoStackPipeline
    period, M = 600.0, 60
    mesh = square_cell(32, radius=120.0 / period)
    wl = np.linspace(400.0, 900.0, batch)
    th = np.radians(1e-5)
    k = 2 * np.pi / wl
    kp = np.stack([k * np.sin(th) * np.cos(th), k * np.sin(th) * np.sin(th)], axis=1)
    g = torch.Generator(device='cuda').manual_seed(0)
    shape = (batch, mesh.nel, M, 13, 3)
    cr = lambda: 0.02 * torch.complex(torch.randn(shape, dtype=torch.float64, device=dev, generator=g),
                                      torch.randn(shape, dtype=torch.float64, device=dev, generator=g))
    s1, s2 = cr(), cr()
    k0 = 2 * np.pi / (wl / period)
    rng = np.random.default_rng(0)
    beta = rng.uniform(0, 2, (batch, M)) * k0[:, None] + 1j * rng.uniform(0, 0.1, (batch, M)) * k0[:, None]
    beta = torch.tensor(beta, device=dev)
    res = {}
    lists = {}
    for prec in ('fp64', 'tf32x3'):
        pl = NanoStackPipeline(mesh, period, 3, M, batch, 100.0, precision=prec)
        pl.load(wl, kp, s1, s2, beta)
        out = pl.capture()
        ms = _timed(pl.replay, steps, warmup=2)
        res[prec] = batch / (ms / 1e3)
        lists[prec] = np.concatenate([out[k].cpu().numpy().reshape(batch, -1)
                                      for k in ('a_list', 't_list', 'r_list')], axis=1)
        del pl
    # plain: one wavelength per call, FP64, eager
    pl1 = NanoStackPipeline(mesh, period, 3, M, 1, 100.0, precision='fp64')
    n_plain = 10
    loads = [(wl[i:i + 1], kp[i:i + 1], s1[i:i + 1].clone(), s2[i:i + 1].clone(), beta[i:i + 1].clone())
             for i in range(n_plain)]

    def plain():
        for a in loads:
            pl1.load(*a)
            pl1.forward()

    ms1 = _timed(plain, 3, warmup=1)
    plain_wl = n_plain / (ms1 / 1e3)
    return {'batched_fp64_wl_per_s': res['fp64'], 'plain_wl_per_s': plain_wl,
            'ratio': res['fp64'] / plain_wl,
            'batched_tf32x3_wl_per_s': res['tf32x3'], 'ratio_tf32x3': res['tf32x3'] / plain_wl,
            'tf32x3_max_abs_delta_RTA_vs_fp64': float(np.abs(lists['tf32x3'] - lists['fp64']).max()),
            'note': 'ratio = the all-FP64 batched chain (meets the 1e-6 bar); ratio_tf32x3 = the chain '
                    'with the tensor-core J, whose a/t/r differ from FP64 by the delta given on these '
                    'random synthetic fields (on the physical modes of the FEM solve see fem_modes)',
            'workload': 'config 1: 1 array (period 600 nm, 2048 triangles, 60 modes, P = 58), '
                        '%d wavelengths 400-900 nm, synthetic seeded mode fields; batched = one CUDA '
                        'graph, FP64 interfaces/cascade; plain = one wavelength per call, FP64, '
                        'eager' % batch}


def config1_physical(dev, batch=50, steps=10):
    """The config-1 chain on physical Bloch modes: the GPU FEM solve
    (emustack_b200.fem) of a 2D array layer on the reference's own test mesh
    (4testing-600_120.mail: period 600 nm, a wire of 120 nm diameter, 518
    triangles) with the config-1 materials (n = 3.5 + 0.01i in 1.46, h = 100
    nm, substrate 1.46, air above), max order 3 (P = 58), 60 Bloch modes, at
    `batch` wavelengths 400-900 nm.  The modes are solved first (not timed);
    then the chain (J / J_dag, normalisation, interfaces, cascade, fluxes) is
    timed as in config1_chain: plain = one wavelength per call, FP64; batched
    = one CUDA graph, with the FP64 and the split-TF32 x3 J.  The modes of the
    wavelengths are solved by 4 host threads at once (fem.solve_pairs)."""
    import torch
    from emustack_b200.fem import FemMesh, FemModeSolver
    from emustack_b200.mesh import Mesh
    from emustack_b200.pipeline import NanoStackPipeline
    period, M, mo = 600.0, 60, 3
    mail = os.path.join(ROOT, 'tests', 'golden', '4testing-600_120.mail')
    mesh = Mesh.from_mail(mail)
    fem = FemModeSolver(FemMesh.from_mesh(mesh))
    wl = np.linspace(400.0, 900.0, batch)
    th = np.radians(1e-5)
    k = 2 * np.pi / wl
    kp = np.stack([k * np.sin(th) * np.cos(th), k * np.sin(th) * np.sin(th)], axis=1)
    n_effs = np.array([1.46, 3.5 + 0.01j])
    t0 = time.perf_counter()
    s1 = torch.empty((batch, mesh.nel, M, 13, 3), dtype=torch.complex128, device=dev)
    s2 = torch.empty_like(s1)
    beta = torch.empty((batch, M), dtype=torch.complex128, device=dev)
    from emustack_b200.fem import solve_pairs
    jobs = [(n_effs, wl[i] / period, kp[i] * period, None) for i in range(batch)]
    for i, (b1, f1, b2, f2) in enumerate(solve_pairs(fem.mesh, jobs, M, workers=4)):
        s1[i], s2[i] = f1, f2
        beta[i] = torch.as_tensor(b1)
    torch.cuda.synchronize()
    fem_s = time.perf_counter() - t0
    res, lists = {}, {}
    for prec in ('fp64', 'tf32x3'):
        pl = NanoStackPipeline(mesh, period, mo, M, batch, 100.0, precision=prec)
        pl.load(wl, kp, s1, s2, beta)
        out = pl.capture()
        ms = _timed(pl.replay, steps, warmup=2)
        res[prec] = batch / (ms / 1e3)
        lists[prec] = np.concatenate([out[k].cpu().numpy().reshape(batch, -1)
                                      for k in ('a_list', 't_list', 'r_list')], axis=1)
        del pl
    pl1 = NanoStackPipeline(mesh, period, mo, M, 1, 100.0, precision='fp64')
    n_plain = 10
    loads = [(wl[i:i + 1], kp[i:i + 1], s1[i:i + 1].clone(), s2[i:i + 1].clone(), beta[i:i + 1].clone())
             for i in range(n_plain)]

    def plain():
        for a in loads:
            pl1.load(*a)
            pl1.forward()

    ms1 = _timed(plain, 3, warmup=1)
    plain_wl = n_plain / (ms1 / 1e3)
    return {'batched_fp64_wl_per_s': res['fp64'], 'plain_wl_per_s': plain_wl, 'ratio': res['fp64'] / plain_wl,
            'batched_tf32x3_wl_per_s': res['tf32x3'], 'ratio_tf32x3': res['tf32x3'] / plain_wl,
            'tf32x3_max_abs_delta_RTA_vs_fp64': float(np.abs(lists['tf32x3'] - lists['fp64']).max()),
            'fem_modes_s': fem_s,
            'workload': 'config 1 chain on physical modes: GPU FEM modes of the reference test mesh '
                        '(518 triangles, 60 modes, P = 58), n = 3.5 + 0.01i in 1.46, h = 100 nm, %d '
                        'wavelengths 400-900 nm' % batch}


def array_pool(n_points, seed=0, period=500.0):
    """Spectral points with two synthetic nanostructured-array layers each
    (ArrayLayer: Bloch k_z and J / J_dag made on the device): P = 2 Npw
    log-uniform in [50, 900] (nearest order set), M = P + 20, wavelength
    U(350, 1100) nm, theta U(0, 60), phi U(0, 90) degrees."""
    import torch
    from emustack_b200.array_serving import ArrayLayer
    rng = np.random.default_rng(seed)
    tab = order_table(period)
    g = torch.Generator(device='cuda').manual_seed(seed)
    pool = []
    for _ in range(n_points):
        mo = int(np.argmin(np.abs(tab - float(np.exp(rng.uniform(np.log(50), np.log(900)))) / 2)))
        P = 2 * int(tab[mo])
        M = P + 20
        wl = float(rng.uniform(350, 1100))
        th, ph = np.radians(rng.uniform(0, 60)), np.radians(rng.uniform(0, 90))
        k = 2 * np.pi / wl
        kp = np.array([k * np.sin(th) * np.cos(ph), k * np.sin(th) * np.sin(ph)])
        k0 = 2 * np.pi / (wl / period)
        cr = lambda *sh: torch.complex(torch.randn(sh, dtype=torch.float64, device='cuda', generator=g),
                                       torch.randn(sh, dtype=torch.float64, device='cuda', generator=g))
        lays = [ArrayLayer(rng.uniform(0, 2, M) * k0 + 1j * rng.uniform(0, 0.1, M) * k0,
                           J=cr(P, M) / np.sqrt(P), J_dag=cr(M, P) / np.sqrt(P)) for _ in range(2)]
        pool.append((mo, wl, kp, lays))
    return pool


def mixed_requests(n, seed, array_frac=0.0, pool=None, period=500.0):
    """n requests in random order: film requests (film_requests) and a
    fraction array_frac of array stacks (film substrate, 2-12 finite layers
    each a film or one of the two array layers of a pool point, air), so
    that requests share layers and the server's interface cache is used."""
    from emustack_b200.array_serving import ArrayRequest
    na = int(round(n * array_frac)) if pool else 0
    reqs = film_requests(n - na, seed, period)
    rng = np.random.default_rng(seed + 7)
    pols = ('TE', 'TM', 'un', 'R Circ')
    for i in range(na):
        mo, wl, kp, lays = pool[int(rng.integers(len(pool)))]
        K = int(rng.integers(2, 13))
        mid = [lays[int(rng.integers(2))] if rng.random() < 0.5
               else complex(rng.uniform(1.3, 4.0), rng.uniform(0, 0.5)) for _ in range(K)]
        reqs.append(ArrayRequest([1.46 + 0j] + mid + [1.0 + 0j], rng.uniform(20, 300, K), wl, kp, period, mo,
                                 pol=pols[i % 4]))
    order = np.random.default_rng(seed + 3).permutation(len(reqs))
    return [reqs[i] for i in order]


def serving_run(rate, seconds=1.0, seed=0, array_frac=0.0, pool=None, n_streams=2):
    """Open-loop Poisson arrivals of uneven requests at `rate` per second
    through the continuous-batching server (GsmServer); latency from each
    request's scheduled arrival to its result on the host.  array_frac > 0
    mixes in array-stack requests built on the layers of `pool`."""
    from emustack_b200.serving import GsmServer
    n = max(int(rate * seconds), 200)
    reqs = mixed_requests(n, seed, array_frac, pool)
    gaps = np.random.default_rng(seed + 1).exponential(1.0 / rate, n)
    srv = GsmServer(max_batch=32768, batching='mixed', n_streams=n_streams).start()
    warm = mixed_requests(max(64, min(32768, int(rate * 0.2))), seed + 2, array_frac, pool)
    for _ in range(2):
        for f in [srv.submit(r) for r in warm]:
            f.result(timeout=300)
    srv.latencies.clear()
    srv.array_latencies.clear()
    c = srv.cache
    c.hits = c.misses = c.evictions = 0
    srv.batch_sizes.clear()
    srv.n_batches = 0
    srv.t_first = srv.t_last = None
    t0 = time.perf_counter() + 0.05
    arrivals = t0 + np.cumsum(gaps)
    futs = []

    def submitter():
        i = 0
        while i < n:
            now = time.perf_counter()
            while i < n and arrivals[i] <= now:
                reqs[i].t_arrival = float(arrivals[i])
                futs.append(srv.submit(reqs[i]))
                i += 1
            if i < n:
                time.sleep(max(2e-4, arrivals[i] - time.perf_counter()))

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
    out = {'offered_per_s': rate, 'requests': n, 'achieved_per_s': st['throughput_per_s'],
           'p50_ms': st['p50_ms'], 'p99_ms': st['p99_ms'], 'batches': st['batches'],
           'mean_batch': st['mean_batch'], 'streams': n_streams,
           'workload': 'config 5: Poisson arrivals of uneven all-film solves (P log-uniform 50-900, '
                       '2-12 layers, mixed polarisations) through GsmServer (host scheduling thread, '
                       'continuous batching); latency from scheduled arrival to host result'}
    if array_frac:
        cs = st['smatrix_cache']
        out.update(array_frac=array_frac, array_requests=st['array_requests'],
                   array_p50_ms=st['array_p50_ms'], array_p99_ms=st['array_p99_ms'],
                   cache_hits=cs['hits'], cache_misses=cs['misses'],
                   workload=out['workload'] + '; a fraction array_frac are array stacks (P 50-900, M = P + 20, '
                   'layers shared across requests through the device interface cache)')
    return out


def ring_serving_run(rate, seconds=1.0, seed=0):
    """Open-loop Poisson arrivals of uneven film requests at `rate` per
    second through the device-resident request loop (DeviceFilmServer: a
    persistent kernel picks requests up from a pinned host ring, no launch
    per request); latency from each request's scheduled arrival to the host
    seeing its completion word."""
    from emustack_b200.serving import DeviceFilmServer
    n = max(int(rate * seconds), 200)
    reqs = [r for r in film_requests(n, seed) if len(r.n) <= 16 and r.npw <= 512]
    n = len(reqs)
    gaps = np.random.default_rng(seed + 1).exponential(1.0 / rate, n)
    srv = DeviceFilmServer(capacity=8192, idle_seconds=1.0)
    try:
        for r in film_requests(256, seed + 2):       # warm the loop
            srv.take(srv.submit(r))
        pending, lat = collections.OrderedDict(), []
        t0 = time.perf_counter() + 0.02
        arrivals = t0 + np.cumsum(gaps)
        gc.collect()
        gc.disable()
        try:
            i = 0
            while i < n or pending:
                now = time.perf_counter()
                j = i
                while j < n and arrivals[j] <= now:
                    j += 1
                if j > i:   # every request that has arrived, in one call
                    for t, a in zip(srv.submit_many(reqs[i:j]), arrivals[i:j]):
                        pending[t] = a
                    i = j
                # the oldest pending tickets (results complete about in order),
                # read in one call; islice keeps each pass bounded
                done = srv.poll_many(list(itertools.islice(pending, 256)))
                now = time.perf_counter()
                for t in done:
                    lat.append(now - pending.pop(t))
                if i < n and not pending:
                    time.sleep(max(0.0, min(1e-4, arrivals[i] - time.perf_counter())))
        finally:
            gc.enable()
        t_end = time.perf_counter()
        srv.stop()
    finally:
        srv.close()
    lat = np.array(lat) * 1e3
    return {'offered_per_s': rate, 'requests': n, 'achieved_per_s': n / (t_end - t0),
            'p50_ms': float(np.percentile(lat, 50)), 'p99_ms': float(np.percentile(lat, 99)),
            'workload': 'config 5: Poisson arrivals of uneven all-film solves (P log-uniform 50-900, '
                        '2-12 layers, mixed polarisations) through the device-resident request loop '
                        '(one persistent kernel, pinned host ring, one warp per request; the client submits '
                        'the requests that have arrived and reads the oldest results with one call each per '
                        'pass); latency from scheduled arrival to the host holding the result'}


def ring_capacity(n=8000, seed=0):
    """The device-resident loop apart from the client's pace: n requests
    submitted back to back, then the time until the last is solved (read
    without reading the others) and the host cost per submit and per read."""
    from emustack_b200 import _lib
    from emustack_b200.serving import DeviceFilmServer
    reqs = [r for r in film_requests(n, seed) if len(r.n) <= _lib.RING_MAX_LAYERS and r.npw <= _lib.RING_MAX_PW]
    srv = DeviceFilmServer(capacity=max(8192, len(reqs) + 1), idle_seconds=2.0)
    try:
        for r in film_requests(256, seed + 2):
            srv.take(srv.submit(r))
        L = _lib.lib()
        t0 = time.perf_counter()
        tickets = [srv.submit(r) for r in reqs]
        t1 = time.perf_counter()
        while L.emu_film_ring_ready(srv._h, tickets[-1]) != 1:
            pass
        t2 = time.perf_counter()
        for t in tickets:
            srv.take(t)
        t3 = time.perf_counter()
        # the same with one call per batch of 512 requests
        t4 = time.perf_counter()
        tickets = []
        for k in range(0, len(reqs), 512):
            tickets += srv.submit_many(reqs[k:k + 512])
        t5 = time.perf_counter()
        while L.emu_film_ring_ready(srv._h, tickets[-1]) != 1:
            pass
        t6 = time.perf_counter()
        got = 0
        for k in range(0, len(tickets), 512):
            part = tickets[k:k + 512]
            while part:
                done = srv.poll_many(part)
                got += len(done)
                part = [t for t in part if t not in done]
        t7 = time.perf_counter()
        assert got == len(tickets)
        srv.stop()
    finally:
        srv.close()
    m = len(reqs)
    return {'requests': m, 'submit_us': (t1 - t0) / m * 1e6, 'read_us': (t3 - t2) / m * 1e6,
            'solved_after_last_submit_ms': (t2 - t1) * 1e3, 'device_rate_at_least_per_s': m / (t2 - t0),
            'batched_submit_us': (t5 - t4) / m * 1e6, 'batched_read_us': (t7 - t6) / m * 1e6,
            'batched_solved_after_last_submit_ms': (t6 - t5) * 1e3,
            'batched_device_rate_at_least_per_s': m / (t6 - t4),
            'workload': 'config 5 requests submitted back to back to the device-resident loop, one call per '
                        'request, then one call per 512 requests'}


def north_star_extras(dev, w, solver, value):
    """The batched / mixed-precision GSM against the plain FP64 GPU GSM, and a
    short serving run (bounded work: about half a minute)."""
    import torch
    out = {'note': 'plain FP64 GPU GSM = this library called once per solve from Python (about '
                   '35 us of host work per call), as the reference calls its GSM once per '
                   'Stack.calc_scat'}
    t0 = time.perf_counter()
    plain2 = plain_config2(dev, w)
    out['config2'] = {'plain_points_per_s': plain2, 'batched_points_per_s': value, 'ratio': value / plain2}
    try:
        out['config1'] = config1_chain(dev)
    except Exception as e:   # report, do not lose the headline line
        out['config1'] = {'error': repr(e)}
    torch.cuda.empty_cache()
    reqs = film_requests(4096, seed=0)
    ms_var, ms_one = time_film_mix(dev, reqs)
    specs = array_stack_specs(96, seed=1)
    ms_ag = time_array_stacks(specs, group=True)
    ms_a1 = time_array_stacks(specs[:12], group=False, n_streams=1) / 12 * len(specs)
    torch.cuda.empty_cache()
    nf, na = len(reqs), len(specs)
    out['config4_mix'] = {
        'films': {'solves': nf, 'batched_per_s': nf / (ms_var / 1e3), 'plain_per_s': nf / (ms_one / 1e3),
                  'ratio': ms_one / ms_var},
        'arrays': {'solves': na, 'batched_per_s': na / (ms_ag / 1e3), 'plain_per_s': na / (ms_a1 / 1e3),
                   'ratio': ms_a1 / ms_ag},
        'mix_50_50': {'ratio': (ms_one / nf + ms_a1 / na) / (ms_var / nf + ms_ag / na)},
        'workload': 'config 4: uneven film solves in one emu_film_var_batch launch vs one launch per '
                    'solve; array stacks (P 50-900, M = P + 20, 2-12 arrays, interfaces included) '
                    'grouped by shape on 4 streams vs one call per stack (samples of 256 and 12, '
                    'extrapolated); mix_50_50 = equal numbers of both'}
    try:
        out['serving'] = serving_run(20000.0, 1.0)
    except Exception as e:
        out['serving'] = {'error': repr(e)}
    try:
        out['serving_device_loop'] = ring_serving_run(20000.0, 1.0)
    except Exception as e:
        out['serving_device_loop'] = {'error': repr(e)}
    torch.cuda.empty_cache()
    try:
        f = fem_line(3)
        out['fem_modes'] = {k: f[k] for k in ('metric', 'value', 'unit', 'ms_per_layer',
                                              'kz_max_rel_err_vs_reference', 'tensor_core_J_on_these_modes',
                                              'cpu_baseline', 'gratings_1d')}
        out['fem_modes']['workload'] = f['config']['workload']
        out['fem_modes']['ratio_vs_cpu_baseline'] = f['value'] / f['cpu_baseline']['value']
    except Exception as e:
        out['fem_modes'] = {'error': repr(e)}
    out['seconds'] = time.perf_counter() - t0
    return out


# ---------------------------------------------------------------- --config N
def config3_line(steps):
    """Config 3 per wavelength: 4 arrays, period 700 nm, max order 10
    (P = 618), M = 400, J + J_dag on the tensor cores from complex64 fields on
    a 20 000-triangle mesh, interfaces and cascade (FP64) for 148
    wavelengths at once."""
    import torch
    from emustack_b200.dense import DenseStackSolver
    from emustack_b200.films import grating_orders
    from emustack_b200.mesh import square_cell
    from emustack_b200.overlap import DeviceMesh, overlap_batch
    dev = torch.device('cuda')
    period, mo, M = 700.0, 10, 400
    mesh = square_cell(100, radius=0.3)
    px, py = grating_orders(mo, period, period)
    g = torch.Generator(device='cuda').manual_seed(0)
    shape = (1, mesh.nel, M, 13, 3)
    cr = lambda: torch.complex(torch.randn(shape, dtype=torch.float32, device=dev, generator=g),
                               torch.randn(shape, dtype=torch.float32, device=dev, generator=g))
    s1, s2 = cr(), cr()
    dm = DeviceMesh(mesh)
    bloch = torch.tensor([[1e-6, 1e-13]], dtype=torch.float64, device=dev)
    k0 = torch.tensor([2 * np.pi / (650.0 / period)], dtype=torch.float64, device=dev)
    ms_j = _timed(lambda: overlap_batch(dm, px, py, mo, bloch, k0, s1, s2, precision='tf32x3'), steps)
    s1, s2 = s1.to(torch.complex128), s2.to(torch.complex128)
    ms_j64 = _timed(lambda: overlap_batch(dm, px, py, mo, bloch, k0, s1, s2, precision='fp64'), max(1, steps // 2),
                    warmup=1)
    del s1, s2
    torch.cuda.empty_cache()
    specs = [dict(mo=mo, npw=len(px), K=4, M=M, wl=float(w), seed=i)
             for i, w in enumerate(np.linspace(400, 900, 148))]
    ms_gsm = time_array_stacks(specs, group=True, n_streams=1)
    return {'config': 3, 'P': 2 * len(px), 'M': M, 'nel': mesh.nel,
            'J_pair_ms_per_layer': ms_j, 'J_pair_fp64_ms_per_layer': ms_j64,
            'interfaces_cascade_ms_per_wavelength': ms_gsm / 148,
            'ms_per_wavelength': 4 * ms_j + ms_gsm / 148}


# ----------------------------------------------------------------- --fields
def fields_line(steps, nel=20000):
    """Field reconstruction from the GSM amplitudes.

    Plane-wave fields (emu_pw_fields): one film layer (the 6th of 12) of 256
    points of the thin-film workload (81 orders per polarisation), on a
    51 x 51 x 4 grid per point (fields_in_plane's grid), against the numpy
    restatement of the reference's loop on a sample.  Bloch-mode node fields
    (emu_bloch_fields_plane): one 2D layer of 20 000 elements and 400 modes
    (the config-3 layer size), against the numpy restatement of
    field_value_plane on 2 000 elements."""
    import torch
    from emustack_b200.fields import bloch_fields_plane, film_batch_fields, pw_fields
    from emustack_b200.films import FilmStackSolver
    from emustack_b200.probe import fp64_peak_tflops
    from oracle import fields_oracle as F
    dev = torch.device('cuda')
    w = workload(seed=0)
    B, L, layer = 256, N_FILMS + 2, 6
    solver = FilmStackSolver(L, MAX_ORDER, PERIOD)
    S = solver.npw
    wl = torch.tensor(w['wl'][:B], device=dev)
    kp = torch.tensor(w['k_pll'][:B], device=dev)
    n = torch.tensor(w['n'][:B], device=dev)
    hs = torch.tensor(w['heights'], device=dev)
    out = solver.solve(wl, kp, n, hs, pol=POL, want=('kz', 'vec_coef', 'sort_order'))
    h_norm = float(w['heights'][layer - 1]) / PERIOD
    r = np.linspace(0.0, 1.0, 51)
    zs = np.linspace(0.0, h_norm, 4)
    # inputs of the kernel, formed once (film_batch_fields forms them per call)
    film_batch_fields(solver, out, kp, n, layer, r, r, zs, heights_nm=hs, grid=True)
    two_pi = 2 * np.pi
    kpn = kp * PERIOD
    alphas = (kpn[:, 0:1] + solver.d_px.to(torch.float64)[None] * two_pi).contiguous()
    betas = (kpn[:, 1:2] + solver.d_py.to(torch.float64)[None] * two_pi).contiguous()
    row = L - 1 - layer
    args = dict(alphas=alphas, betas=betas, sort_order=out['sort_order'].clone(),
                kz=out['kz'][:, layer].contiguous(), n=n[:, layer].contiguous(),
                vec_coef_down=out['vec_coef_down'][:, row].contiguous(),
                vec_coef_up=out['vec_coef_up'][:, row].contiguous(),
                x=torch.tensor(r, device=dev), y=torch.tensor(r, device=dev), z=torch.tensor(zs, device=dev),
                height_norm=torch.full((B,), h_norm, dtype=torch.float64, device=dev), grid=True)
    Q = 51 * 51 * 4
    ms = _timed(lambda: pw_fields(**args), steps, warmup=3)
    terms = B * Q * S
    # CPU: the restatement of the reference's per-point loop on 2 points x 11 x 11 x 4
    a = {k: (v.cpu().numpy() if hasattr(v, 'cpu') else v) for k, v in args.items()}
    rs = np.linspace(0.0, 1.0, 11)
    t0 = time.perf_counter()
    for b in range(2):
        F.pw_field_grid(a['alphas'][b], a['betas'][b], a['sort_order'][b], a['kz'][b], a['n'][b],
                        a['vec_coef_down'][b], a['vec_coef_up'][b], rs, rs, zs, height_norm=h_norm)
    cpu_s = time.perf_counter() - t0
    cpu_pts = 2 * 11 * 11 * 4 / cpu_s
    # the grid path: per (x, y) point and order one complex product X Y (6 FP64 operations),
    # per z value three complex multiply-adds (8 each); the per-axis tables are not counted
    flops_per_term = 24 + 6.0 / len(zs)
    pw = {'stacks': B, 'points_per_stack': Q, 'orders': S, 'ms': ms,
          'field_points_per_s': B * Q / (ms / 1e3), 'order_terms_per_s': terms / (ms / 1e3),
          'cpu_field_points_per_s': cpu_pts, 'cpu_sample': '2 stacks x 11 x 11 x 4 points, numpy, 1 core',
          'fp64_peak_tflops': fp64_peak_tflops(),
          'path': 'grid: per-axis exponential tables (emu_pw_fields workspace), then a contraction over orders',
          'note': 'fp64_tflops counts the contraction (24 + 6 / nz FP64 operations per term)'}
    pw['fp64_tflops'] = terms * flops_per_term / (ms / 1e3) / 1e12
    pw['frac'] = pw['fp64_tflops'] / pw['fp64_peak_tflops']
    del out, args
    torch.cuda.empty_cache()
    # Bloch-mode node fields at the config-3 layer size (nel = 20 000)
    M = 400
    g = torch.Generator(device='cuda').manual_seed(0)
    sol = torch.complex(torch.randn((1, nel, M, 13, 3), dtype=torch.float64, device=dev, generator=g),
                        torch.randn((1, nel, M, 13, 3), dtype=torch.float64, device=dev, generator=g))
    kz = torch.complex(torch.rand((1, M), dtype=torch.float64, device=dev, generator=g) * 3 + 0.5,
                       torch.rand((1, M), dtype=torch.float64, device=dev, generator=g) * 0.5)
    vc = torch.complex(torch.randn((1, 2 * M), dtype=torch.float64, device=dev, generator=g),
                       torch.randn((1, 2 * M), dtype=torch.float64, device=dev, generator=g))
    msb = _timed(lambda: bloch_fields_plane(sol, kz, vc, 0.5, 0.2), steps, warmup=3)
    bytes_alg = nel * M * 18 * 16 + 2 * M * 16 + M * 16 + nel * 18 * 16
    hbm, hbm_src = hbm_peak()
    ns = min(2000, nel)
    sol_s = sol[0, :ns].cpu().numpy()
    kz_h, vc_h = kz[0].cpu().numpy(), vc[0].cpu().numpy()
    t0 = time.perf_counter()
    F.bloch_field_plane(sol_s, kz_h, vc_h, 0.5, 0.2)
    cpu_b = time.perf_counter() - t0
    bl = {'elements': nel, 'modes': M, 'ms': msb, 'elements_per_s': nel / (msb / 1e3),
          'achieved_gbs': bytes_alg / (msb / 1e3) / 1e9, 'peak_gbs': hbm, 'peak_source': hbm_src,
          'frac': bytes_alg / (msb / 1e3) / 1e9 / hbm, 'algorithmic_bytes': bytes_alg,
          'cpu_elements_per_s': ns / cpu_b, 'cpu_sample': '%d elements, numpy, 1 core' % ns}
    return {'workload': 'fields', 'pw_fields': pw, 'bloch_fields_plane': bl}


def fem_tc_delta(modes, fx, key):
    """J / J_dag of the FEM modes by the FP64 and the split-TF32 x3 tensor-core
    contraction, each through the drop-in Stack of the reference's test case 1
    (SiO2 substrate, the 2330 nm wire layer, air): the largest differences of
    R_net and of the a/t/r lists between the two."""
    from emustack_b200 import materials, objects
    from emustack_b200.mesh import Mesh
    from emustack_b200.stack import Stack
    gold = np.load(os.path.join(ROOT, 'tests', 'golden', 'case_1.npz'), allow_pickle=True)
    b1, s1, b2, s2 = modes
    per = float(gold['p0_period'])
    light = objects.Light(float(gold['p0_wl_nm']), max_order_PWs=int(fx[key + 'max_order']), theta=0.0, phi=0.0)
    n_effs = fx[key + 'n_effs']
    mesh = Mesh.from_mail(os.path.join(ROOT, 'tests', 'golden', '4testing-600_120.mail'))
    ns = objects.NanoStruct('2D_array', per, 120, height_nm=float(gold['p0_heights_nm'][0]),
                            background=materials.Material(complex(n_effs[0])),
                            inclusion_a=materials.Material(complex(n_effs[1])), loss=True, mesh=mesh)
    films = [objects.ThinFilm(period=per, height_nm='semi_inf', material=materials.Material(complex(gold[k])),
                              loss=False) for k in ('p0_lay0_n', 'p0_lay2_n')]
    res = {}
    for prec in ('fp64', 'tf32x3'):
        sim = ns.calc_modes(light, k_z=b1, fields={'sol1': s1, 'sol2': s2, 'beta1': b1, 'mesh': mesh,
                                                    'precision': prec})
        st = Stack((films[0].calc_modes(light), sim, films[1].calc_modes(light)))
        st.calc_scat(pol='TE')
        flat = np.concatenate([np.ravel(np.asarray(v, dtype=complex)).real
                               for lst in (st.a_list, st.t_list, st.r_list) for v in lst])
        res[prec] = (np.asarray(st.R_net), flat)
    return {'max_abs_delta_R_net': float(np.abs(res['tf32x3'][0] - res['fp64'][0]).max()),
            'max_abs_delta_RTA': float(np.abs(res['tf32x3'][1] - res['fp64'][1]).max()),
            'stack': 'reference test case 1 at 500 nm (SiO2 / 40-mode wire layer / air), TE'}


def fem_line(steps, concurrent=True):
    """FEM Bloch-mode solve of one nanostructured layer on the GPU (row f1).

    Workload: the reference's own test mesh 4testing-600_120.mail (518 P2
    triangles, 6 216 DOFs; a 120 nm Si_c wire in air at period 600 nm), the
    inputs the reference passes to its solver for test case 1 at 500 nm (40
    Bloch modes, tests/golden/fem.npz): one layer = the prime and the adjoint
    solve (element matrices, assembly, LU and inverse of K - shift M, block
    Krylov-Schur, nodal fields), timed host to host (the projected
    eigenproblem is reduced on the host).  CPU baseline: the oracle's
    restatement (scipy ARPACK on a SuperLU factorisation) on one solve."""
    import torch
    from emustack_b200.fem import FemMesh, FemModeSolver
    from emustack_b200.probe import fp64_peak_tflops
    from oracle import fem_oracle as F
    gold = os.path.join(ROOT, 'tests', 'golden')
    mail = os.path.join(gold, '4testing-600_120.mail')
    fx = np.load(os.path.join(gold, 'fem.npz'))
    ref_kz = np.load(os.path.join(gold, 'case_1.npz'), allow_pickle=True)['p0_lay1_k_z']
    key = 'case1_p0_'
    n_effs, wl_norm = fx[key + 'n_effs'], float(fx[key + 'wl_norm'])
    bloch, nval = np.asarray(fx[key + 'k_pll_norm'], float), int(fx[key + 'num_BMs'])
    shift = complex(fx[key + 'shift']).real
    mesh = FemMesh.from_mail(mail)
    solver = FemModeSolver(mesh)
    k0 = 2 * np.pi / wl_norm

    def layer():
        return solver.solve_pair(n_effs, wl_norm, bloch, nval, shift=shift, concurrent=concurrent)

    for _ in range(2):
        out = layer()
    torch.cuda.synchronize()
    times = []
    for _ in range(max(3, steps)):
        t0 = time.perf_counter()
        out = layer()
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    ms = 1e3 * float(np.median(times))
    kz_err = float(np.max(np.abs(out[0] - ref_kz) / np.abs(ref_kz)))
    tc = fem_tc_delta(out, fx, key)
    # parts of one solve (CUDA events around the device steps)
    n = mesh.neq
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record()
    solver.factor(n_effs, k0, bloch, shift)
    ev[1].record()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    solver.eigs(nval)
    torch.cuda.synchronize()
    eig_ms = 1e3 * (time.perf_counter() - t0)
    st = dict(solver.stats)
    blk = solver.block
    X = torch.randn(n, blk, dtype=torch.complex128, device='cuda')
    Y = torch.empty_like(X)
    apply_ms = _timed(lambda: solver.apply(X, Y), 10, warmup=3)
    del solver.Ainv
    nt = len(mesh.trows)
    lu_flops = 8.0 / 3.0 * n ** 3
    inv_flops = 8.0 * n ** 2 * nt
    factor_ms = ev[0].elapsed_time(ev[1])
    # CPU: the oracle's solve of the prime modes
    x, tn, tab, tel = F.read_mail(mail)
    t0 = time.perf_counter()
    F.solve_modes(x, tn, tab, tel, n_effs, wl_norm, bloch, nval, shift=shift)
    cpu_s = (time.perf_counter() - t0) / 2.0    # solve_modes does the prime and the adjoint solve
    peak = fp64_peak_tflops()
    hbm, hbm_src = hbm_peak()
    g1d = fem1d_part(steps, concurrent)
    return {
        'metric': 'FEM layer solves/s (prime + adjoint Bloch modes)', 'value': 1e3 / ms, 'unit': 'layers/s',
        'ms_per_layer': ms, 'steps': max(3, steps), 'dtype': 'c128',
        'prime_and_adjoint': 'concurrent (two streams, two host threads)' if concurrent else 'one after the other',
        'config': {'workload': 'reference test mesh 4testing-600_120.mail, 518 P2 triangles, %d DOFs, '
                               '%d Bloch modes, test case 1 at 500 nm' % (n, nval)},
        'kz_max_rel_err_vs_reference': kz_err,
        'tensor_core_J_on_these_modes': tc,
        'solve_parts': {'element_matrices_assembly_lu_inverse_ms': factor_ms, 'krylov_schur_ms': eig_ms,
                        'krylov_stats': st, 'operator_apply_ms': apply_ms, 'vectors_per_apply': blk},
        'roofline': {'lu_and_inverse_tflops': (lu_flops + inv_flops) / (factor_ms / 1e3) / 1e12,
                     'fp64_peak_tflops': peak, 'frac': (lu_flops + inv_flops) / (factor_ms / 1e3) / 1e12 / peak,
                     'operator_gbs': 16.0 * n * nt / (apply_ms / 1e3) / 1e9, 'hbm_peak_gbs': hbm,
                     'hbm_source': hbm_src,
                     'note': 'factor time includes the element matrices and assembly (small); complex LU '
                             '8/3 n^3, the nt columns of the inverse from the LU 8 n^2 nt real flops (nt '
                             'transverse DOFs, where M has entries); the operator streams those columns '
                             '(16 n nt bytes) once per block of vectors'},
        'cpu_baseline': {'value': 1.0 / (2 * cpu_s), 'unit': 'layers/s', 'cores': 1, 'kind': 'port',
                         'sample': 'one prime and one adjoint solve of the same layer by the oracle (scipy '
                                   'ARPACK on SuperLU, numpy assembly)'},
        'gratings_1d': g1d,
    }


def fem_holes_line(steps):
    """FEM Bloch-mode solve of a larger layer: the gold film with 266 nm
    square holes at period 940 nm of the reference's test case 5 on its mesh
    4testing-940_266_sq.mail (2 528 P2 triangles, 30 336 DOFs), 100 Bloch
    modes at 1043.4 nm and 5 degrees (the inputs the reference passes,
    tests/golden/fem.npz).  One layer = prime + adjoint solve, timed host to
    host after one untimed layer; CPU baseline: the oracle's prime solve
    (scipy ARPACK on SuperLU) on one host core, doubled for a layer."""
    import torch
    from emustack_b200.fem import FemMesh, FemModeSolver
    from emustack_b200.probe import fp64_peak_tflops
    from oracle import fem_oracle as F
    gold = os.path.join(ROOT, 'tests', 'golden')
    mail = os.path.join(gold, '4testing-940_266_sq.mail')
    fx = np.load(os.path.join(gold, 'fem.npz'))
    ref = np.load(os.path.join(gold, 'case_5.npz'), allow_pickle=True)['p0_lay1_k_z']
    key = 'case5_p0_'
    n_effs, wl_norm = fx[key + 'n_effs'], float(fx[key + 'wl_norm'])
    bloch, nval = np.asarray(fx[key + 'k_pll_norm'], float), int(fx[key + 'num_BMs'])
    shift = complex(fx[key + 'shift']).real
    mesh = FemMesh.from_mail(mail)
    solver = FemModeSolver(mesh)
    solver.solve_pair(n_effs, wl_norm, bloch, nval, shift=shift)
    torch.cuda.synchronize()
    times = []
    for _ in range(max(1, steps)):
        t0 = time.perf_counter()
        out = solver.solve_pair(n_effs, wl_norm, bloch, nval, shift=shift)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    s_layer = float(np.median(times))
    kz_err = float(np.max(np.abs(out[0] - ref) / np.abs(ref)))
    n, nt = mesh.neq, len(mesh.trows)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record()
    solver.factor(n_effs, 2 * np.pi / wl_norm, bloch, shift)
    ev[1].record()
    torch.cuda.synchronize()
    factor_ms = ev[0].elapsed_time(ev[1])
    del solver.Ainv
    torch.cuda.empty_cache()
    flops = 8.0 / 3.0 * n ** 3 + 8.0 * n ** 2 * nt
    peak = fp64_peak_tflops()
    x, tn, tab, tel = F.read_mail(mail)
    t0 = time.perf_counter()
    topo = F.Topology(x, tn, tab)
    K, M = F.element_matrices(topo, x, n_effs, tel, 2 * np.pi / wl_norm, bloch)
    Kg, Mg = F.assemble(topo, K, M)
    F.eigen_solve(Kg, Mg, nval, shift)
    cpu_s = time.perf_counter() - t0
    return {
        'metric': 'FEM layer solves/s (prime + adjoint Bloch modes)', 'value': 1.0 / s_layer, 'unit': 'layers/s',
        's_per_layer': s_layer, 'steps': max(1, steps), 'dtype': 'c128',
        'config': {'workload': 'reference test mesh 4testing-940_266_sq.mail, 2528 P2 triangles, %d DOFs, '
                               '%d Bloch modes, test case 5 (gold film with square holes) at 1043.4 nm' % (n, nval)},
        'kz_max_rel_err_vs_reference': kz_err, 'krylov_stats': dict(solver.stats),
        'factor_ms': factor_ms, 'lu_and_inverse_tflops': flops / (factor_ms / 1e3) / 1e12,
        'fp64_peak_tflops': peak, 'frac': flops / (factor_ms / 1e3) / 1e12 / peak,
        'max_memory_gb': torch.cuda.max_memory_allocated() / 1e9,
        'cpu_baseline': {'value': 1.0 / (2 * cpu_s), 'unit': 'layers/s', 'cores': 1, 'kind': 'port',
                         'sample': 'the oracle\'s prime solve of the same layer (scipy ARPACK on SuperLU), '
                                   'doubled for prime + adjoint'},
    }

def fem1d_part(steps, concurrent=True):
    """The 1D FEM solve of the two gratings of the reference's test case 4
    (period 760 nm, 800 nm, tests/golden/fem1d.npz: the meshes and solver
    inputs the reference passes, the centre inclusion given the width of
    its stored run): one layer = prime + adjoint solve, timed host to host,
    k_z against the reference's stored values, and the oracle's solve
    (scipy ARPACK on SuperLU) of the same layer on one host core."""
    import torch
    from emustack_b200.fem import FemMesh1D, FemModeSolver
    from oracle import fem1d_oracle as F1
    gold = os.path.join(ROOT, 'tests', 'golden')
    fx = np.load(os.path.join(gold, 'fem1d.npz'))
    case4 = np.load(os.path.join(gold, 'case_4.npz'), allow_pickle=True)
    out = {}
    for i in (1, 2):
        p = 'g%d_' % i
        tab = fx[p + 'table_nod'].astype(np.int64).T
        x = fx[p + 'x_arr']
        tel = fx[p + 'type_el'].astype(np.int64).copy()
        tel[(tel == 2) & (np.abs(x[tab[:, 0] - 1] - 0.37) < 1e-9)] = 1
        bloch = [float(fx[p + 'kx']), float(fx[p + 'ky'])]
        wln, nval = float(fx[p + 'wl_norm']), int(fx[p + 'num_BMs'])
        shift = complex(fx[p + 'shift']).real
        n_effs = fx[p + 'n_effs']
        mesh = FemMesh1D(x, tab, tel)
        solver = FemModeSolver(mesh)

        def layer():
            return solver.solve_pair(n_effs, wln, bloch, nval, shift=shift, concurrent=concurrent)

        for _ in range(2):
            res = layer()
        torch.cuda.synchronize()
        times = []
        for _ in range(max(3, steps)):
            t0 = time.perf_counter()
            res = layer()
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
        ms = 1e3 * float(np.median(times))
        ref = case4['p0_lay%d_k_z' % i]
        t0 = time.perf_counter()
        F1.solve_modes(x, tab, tel, n_effs, wln, bloch[0], bloch[1], nval, shift)
        cpu_s = time.perf_counter() - t0
        out['grating_%d' % i] = {
            'elements': int(len(tab)), 'dofs': int(mesh.neq), 'modes': nval, 'ms_per_layer': ms,
            'layers_per_s': 1e3 / ms, 'kz_max_rel_err_vs_reference': float(np.max(np.abs(res[0] - ref) / np.abs(ref))),
            'krylov_stats': dict(solver.stats),
            'cpu_baseline': {'value': 1.0 / cpu_s, 'unit': 'layers/s', 'cores': 1, 'kind': 'port',
                             'sample': 'the oracle\'s prime and adjoint solve of the same grating'}}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--config', type=int, default=2, choices=[1, 2, 3, 4, 5])
    ap.add_argument('--no-extras', action='store_true', help='skip the north_star comparison keys')
    ap.add_argument('--fields', action='store_true',
                    help='time the field reconstruction kernels instead of the GSM')
    ap.add_argument('--fields-elements', type=int, default=20000,
                    help='elements of the nanostructured layer in --fields (a smaller layer for profiling)')
    ap.add_argument('--physical', action='store_true',
                    help='with --config 1: the chain on the GPU FEM modes of a real layer')
    ap.add_argument('--fem', action='store_true',
                    help='time the FEM Bloch-mode solve of a nanostructured layer instead of the GSM')
    ap.add_argument('--fem-holes', action='store_true',
                    help='time the FEM solve of the 30 336-DOF gold-hole layer of the reference\'s case 5')
    ap.add_argument('--fem-sequential', action='store_true',
                    help='with --fem: the prime and adjoint solves one after the other on one stream')
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

    if args.fields:
        print(json.dumps(fields_line(max(args.steps, 5), args.fields_elements)))
        return
    if args.fem:
        print(json.dumps(fem_line(min(args.steps, 10), concurrent=not args.fem_sequential)))
        return
    if args.fem_holes:
        print(json.dumps(fem_holes_line(min(args.steps, 3))))
        return

    if args.config != 2:
        import torch
        dev = torch.device('cuda')
        if args.config == 1 and args.physical:
            print(json.dumps(dict(config1_physical(dev, steps=args.steps), config=1)))
        elif args.config == 1:
            print(json.dumps(dict(config1_chain(dev, steps=args.steps), config=1)))
        elif args.config == 3:
            print(json.dumps(config3_line(args.steps)))
        elif args.config == 4:
            reqs = film_requests(4096, seed=0)
            ms_var, ms_one = time_film_mix(dev, reqs, per_solve=512)
            specs = array_stack_specs(512, seed=1)
            ms_ag = time_array_stacks(specs, group=True)
            ms_a1 = time_array_stacks(specs[:32], group=False, n_streams=1) / 32 * len(specs)
            print(json.dumps({'config': 4, 'film_solves': len(reqs), 'film_batched_ms': ms_var,
                              'film_per_solve_ms': ms_one, 'array_stacks': len(specs),
                              'array_grouped_ms': ms_ag, 'array_per_call_ms': ms_a1}))
        else:
            for r in (1000.0, 10000.0, 100000.0):
                print(json.dumps(dict(serving_run(r, 2.0), config=5)), flush=True)
            for r in (1000.0, 10000.0, 50000.0, 100000.0):
                print(json.dumps(dict(ring_serving_run(r, 2.0), config=5)), flush=True)
            print(json.dumps(dict(ring_capacity(), config=5)), flush=True)
            pool = array_pool(32, seed=11)
            for r, frac in ((10000.0, 0.01), (150.0, 0.5)):
                print(json.dumps(dict(serving_run(r, 2.0, array_frac=frac, pool=pool, n_streams=4), config=5)),
                      flush=True)
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
        args.no_extras = True
    res = run_ours(args, rank, world, local_rank)
    if rank == 0:
        res['cpu_baseline'] = cpu
        print(json.dumps(res))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
