"""Benchmark: CSM + steered-response map throughput (grid-pts x bins / s) on B200.

Workload (one step): the 256-mic precision workload -- 10 s of float32 samples at 51.2 kHz
(512,000 x 256, resident in HBM), CSM with block 1024 / Hanning / 50 % for all 513 bins (999
windows), then the map of every bin on a 401 x 401 grid ('true level', diagonal removed):
160,801 x 513 = 8.25e7 grid-pts x bins per step.

``value``  = grid-pts x bins per second of the whole step (CSM + map), inputs resident on the GPU,
             timed with CUDA events between barriers; max over ranks; each rank runs one full
             instance (weak scaling, no collective on the data path).
``e2e``    = same metric through the public API (``PowerSpectra`` + ``BeamformerBase.result[:]``)
             from pinned host samples to the host result array, copies included.
``--impl reference`` times the CPU oracle (a C/OpenMP port of the reference's numba kernels) on a
bounded sample of the same workload on all host cores.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = 'map grid-pts*bins/s (CSM + map, 256 mics, 401x401 grid, 513 bins)'
UNIT = 'grid-pts*bins/s'
# DRAM bytes of one tensor-core map launch per bin of the 256-mic workload (ncu capture of 4 bins:
# dram__bytes_read.sum + dram__bytes_write.sum, divided by 4)
# DRAM bytes (read + write) of one tensor-core map launch per bin of the 256-mic workload: ncu
# dram__bytes_read.sum + dram__bytes_write.sum of the whole 513-bin launch, divided by 513 (writes still
# in L2 at the kernel's end not counted); split BF16 reads the same R' bytes as TF32
TC_TRAFFIC_PER_BIN = {'fp16': 762.7e6 / 513, 'tf32': 913.5e6 / 513, 'bf16x3': 913.5e6 / 513}
TC_PREC_INDEX = {'bf16x3': 0, 'tf32': 1, 'fp16': 2}
TC_DTYPE = {'tf32': 'tf32 / f32 accum', 'bf16x3': 'bf16x3 (split) / f32 accum',
            'fp16': 'fp16 (R\' scaled per bin) / f32 accum'}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--form', default=None, choices=['tc', 'f64'])
    ap.add_argument('--steer', default='true level')
    ap.add_argument('--no-e2e', action='store_true')
    ap.add_argument('--no-cpu', action='store_true')
    ap.add_argument('--bins', type=int, default=0, help='limit the number of map bins (profiling only)')
    ap.add_argument('--workload', default='precision256',
                    choices=['precision256', 'batched64', 'large3d', 'serving', 'serving-mixed', 'eig', 'damas',
                             'cleansc', 'stream'])
    # FP16 operands (each bin's R' scaled by a power of two) carry TF32's 11-bit significand at half the MMA
    # chain and half the tile bytes: the same error as TF32, the fastest form
    ap.add_argument('--tc-precision', default='fp16', choices=['bf16x3', 'tf32', 'fp16'])
    ap.add_argument('--duration', type=float, default=10.0, help='serving: seconds of offered load')
    ap.add_argument('--no-extra', action='store_true',
                    help='skip the other configurations\' blocks of the default line (profiling runs)')
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons during the timed region: one nvidia-smi process sampling every
    100 ms (-lms), started before the region (its first sample awaited, up to 2 s) and stopped after it."""

    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self._proc = None
        self._t = None
        self._first = threading.Event()

    def _read(self):
        for line in self._proc.stdout:
            parts = [x.strip() for x in line.strip().split(',')]
            if len(parts) >= 5:
                self.rows.append(parts)
                self._first.set()

    def __enter__(self):
        try:
            self._proc = subprocess.Popen(['nvidia-smi', f'--id={self.gpu}', f'--query-gpu={self.FIELDS}',
                                           '--format=csv,noheader,nounits', '-lms', '100'],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:   # clocks are advisory
            self._proc = None
            return self
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()
        self._first.wait(2.0)
        self.rows.clear()   # samples before the timed region starts do not count
        return self

    def __exit__(self, *a):
        if self._proc is None:
            return
        self._proc.terminate()   # the sampler this object started, by its own handle
        try:
            self._proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self._proc.kill()
            self._proc.wait(timeout=5)
        self._t.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['unavailable']}
        sm = [float(r[1]) for r in self.rows if r[1].replace('.', '').isdigit()]
        smax = [float(r[2]) for r in self.rows if r[2].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == 'Active'})
        pw = [float(r[3]) for r in self.rows if r[3].replace('.', '').isdigit()]
        return {'sm_mhz': float(np.median(sm)) if sm else None, 'sm_max_mhz': max(smax) if smax else None,
                'reasons': reasons, 'power_w_max': max(pw) if pw else None, 'samples': len(self.rows)}


def dist_setup(args):
    import torch
    ws = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if args.impl == 'ours':
        torch.cuda.set_device(local)
    if ws > 1:
        import datetime

        import torch.distributed as dist
        backend = 'nccl' if args.impl == 'ours' else 'gloo'
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device='cuda' if dist.get_backend() == 'nccl' else 'cpu')
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def peaks():
    p = ROOT / 'MEASURED_PEAKS.json'
    if p.exists():
        d = json.loads(p.read_text())
        return {'hbm_gbs': d.get('hbm_gbs', 6650.0), 'bf16_tflops': d.get('bf16_tflops', 1590.0),
                'bf16_tflops_sustained': d.get('bf16_tflops_sustained', 1400.0), 'source': 'measured'}
    return {'hbm_gbs': 6650.0, 'bf16_tflops': 1590.0, 'bf16_tflops_sustained': 1400.0, 'source': 'fallback'}


def gemm_peaks(dev, n: int = 8192) -> dict:
    """FP64 (DGEMM) and TF32 (FP32 GEMM with TF32 math) cuBLAS throughput measured here over about half a
    second each (the map launches it is compared with run ~0.1 s): the denominators of the plain form's and
    of the TF32 form's roofline (the peak file holds HBM and BF16 only)."""
    import torch
    out = {}
    for name, dt, tf32, reps in (('fp64_tflops', torch.float64, False, 16), ('tf32_tflops', torch.float32, True, 400)):
        prev = torch.backends.cuda.matmul.allow_tf32
        torch.backends.cuda.matmul.allow_tf32 = tf32
        a = torch.randn((n, n), dtype=dt, device=dev)
        b = torch.randn((n, n), dtype=dt, device=dev)
        c = a @ b
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            torch.matmul(a, b, out=c)
        e1.record()
        torch.cuda.synchronize()
        out[name] = 2.0 * n ** 3 * reps / (e0.elapsed_time(e1) / 1e3) / 1e12
        torch.backends.cuda.matmul.allow_tf32 = prev
        del a, b, c
    out['how'] = f'torch.matmul {n}x{n}x{n}, 16 (FP64) / 400 (TF32) back-to-back reps, CUDA events, this run'
    return out


def host_info() -> dict:
    """Host cores, CPU model and C library of the machine the CPU baselines run on."""
    import platform
    model = None
    try:
        for ln in Path('/proc/cpuinfo').read_text().splitlines():
            if ln.startswith('model name'):
                model = ln.split(':', 1)[1].strip()
                break
    except OSError:
        pass
    return {'nproc': os.cpu_count(), 'threads_available': len(os.sched_getaffinity(0)), 'cpu_model': model,
            'libc': ' '.join(platform.libc_ver())}


# Map bins of the CPU sample: a spread over the band, so that the C library's cosf/sinf cost (which
# grows with the phase argument) is averaged the same way in both arms.
CPU_SAMPLE_BINS = (100, 256, 400)


class CpuSample:
    """The CPU oracle (C/OpenMP port of the reference's numba calcCSM and _freqBeamformer_FullCSM) on a
    bounded sample of the 256-mic workload, on all host threads.  One step is one pass over the sample
    bins ``CPU_SAMPLE_BINS``: per bin the map over the full grid plus one bin's share of the CSM (the Welch
    accumulation of 65 windows over all bins, scaled by K / 65 / F).  ``value`` = grid points / (map time +
    CSM share) per bin, averaged over the pass, so every step weighs the bins alike (the C library's
    cosf/sinf cost grows with the phase argument).  The bench line's ``cpu_baseline`` and the
    ``--impl reference`` arm both use this class, with one warm-up step each."""

    def __init__(self, wl, steer):
        from acoular_b200 import device as D
        from oracle import oracle as O
        self.O = O
        self.ncores = len(os.sched_getaffinity(0))
        O.set_num_threads(self.ncores)
        self.wl, self.steer = wl, steer
        self.M, self.G, self.N = wl.mics.num_mics, wl.grid.size, wl.block_size
        self.F = self.N // 2 + 1
        self.K = D.num_windows(wl.num_samples, self.N, 2)
        self.r0 = O.apparent_r(wl.grid.pos)
        self.rm = O.apparent_r(wl.grid.pos, wl.mics.pos)
        rng = np.random.RandomState(1)
        X = rng.randn(2 * self.M, self.M) + 1j * rng.randn(2 * self.M, self.M)
        self.csm_bin = (X.conj().T @ X) / (2 * self.M)
        self.freqs = O.fftfreq(self.N, wl.fs)
        self.data = rng.randn(64 * (self.N // 2) + self.N, self.M)   # 65 windows; values do not change the cost
        self.norm = O.sig_loss_norm(True, self.M)
        O.beamformer_freq(steer, True, 1.0, self.r0[:64], self.rm[:64], 1.0, self.csm_bin)   # warm the pool

    def step(self) -> float:
        """One pass over the sample bins; returns seconds per bin (the bin's equivalent time)."""
        O, wl = self.O, self.wl
        total = 0.0
        for b in CPU_SAMPLE_BINS:
            t0 = time.perf_counter()
            O.beamformer_freq(self.steer, True, self.norm, self.r0, self.rm, 2 * np.pi * self.freqs[b] / wl.c,
                              self.csm_bin)
            t1 = time.perf_counter()
            O.calc_csm(self.data, self.N, 'Hanning', '50%', 'complex128')
            t2 = time.perf_counter()
            total += (t1 - t0) + (t2 - t1) * (self.K / 65.0) / self.F
        return total / len(CPU_SAMPLE_BINS)

    def describe(self, nsteps: int) -> str:
        return (f'{nsteps} x {len(CPU_SAMPLE_BINS)} bins {list(CPU_SAMPLE_BINS)} (after one warm-up pass), each the map of '
                f'the bin over {self.G} grid points + the CSM of 65 windows x all {self.F} bins scaled to one bin\'s '
                f'share K/65/F, K = {self.K}; C/OpenMP port of the reference numba calcCSM and '
                f'_freqBeamformer_FullCSM, {self.ncores} threads')


def run_reference(args, wl):
    """CPU arm: the oracle port of the reference's CPU path, bounded sample per step (:class:`CpuSample`)."""
    ws = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return
    cs = CpuSample(wl, args.steer)
    cs.step()   # one warm-up pass, as cpu_baseline_sample does
    dt = sum(cs.step() for _ in range(args.steps)) / args.steps
    value = cs.G / dt
    line = {'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': ws, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': dt * 1e3, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic (seeded monopoles)',
            'config': {'workload': wl.name, 'mics': cs.M, 'grid_points': cs.G, 'bins': cs.F, 'block_size': cs.N,
                       'steer_type': args.steer, 'r_diag': True},
            'cpu_baseline': {'value': value, 'unit': UNIT, 'cores': cs.ncores, 'kind': 'port',
                             'sample': cs.describe(args.steps)},
            'host': host_info(),
            'e2e': {'value': value, 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline_sample(wl, steer, nsteps: int = 2):
    """Oracle timing on the host cores for the bench line's cpu_baseline (rank 0, N=1): the same sample
    as the reference arm, one warm-up pass and two timed passes over the sample bins."""
    cs = CpuSample(wl, steer)
    cs.step()
    dt = sum(cs.step() for _ in range(nsteps)) / nsteps
    return {'value': cs.G / dt, 'unit': UNIT, 'cores': cs.ncores, 'kind': 'port', 'sample': cs.describe(nsteps),
            'host': host_info()}


def _line(metric, value, unit, ms, args, config, **extra):
    d = {'metric': metric, 'value': value, 'unit': unit, 'n_gpus': 1, 'steps': args.steps, 'warmup': args.warmup,
         'ms_per_step': ms, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
         'data': 'synthetic (seeded monopoles)', 'config': config}
    d.update(extra)
    print(json.dumps(d), flush=True)


def _err_vs(got: np.ndarray, ref: np.ndarray) -> dict:
    """max / rms of |got - ref| / max|ref| per row (bin) and the L_p difference at each row's peak."""
    got, ref = np.atleast_2d(got), np.atleast_2d(ref)
    err = np.abs(got - ref) / np.abs(ref).max(axis=1, keepdims=True)
    lp = lambda x: 10 * np.log10(np.maximum(x / 4e-10, np.finfo(np.float64).eps))  # noqa: E731
    pk = ref.argmax(axis=1)
    rows = np.arange(ref.shape[0])
    return {'max_rel_err': float(err.max()), 'rms_rel_err': float(np.sqrt((err ** 2).mean())),
            'peak_level_err_db': float(np.abs(lp(got[rows, pk]) - lp(ref[rows, pk])).max())}


def batched_block(steps, warmup, precision):
    """64 uneven instances: per-instance CSM of 30 bins (complex64) + one batched tensor-core map, as one
    CUDA graph.  Accuracy: three instances' maps against the plain FP64 form on the same CSMs."""
    import torch

    from acoular_b200 import device as D
    from acoular_b200 import workloads
    from acoular_b200.batch import BatchPlan, Instance
    dev = torch.device('cuda', 0)
    wls = workloads.batched_instances()
    insts = []
    for wl in wls:
        x = workloads.monopole_time_data_torch(wl, device=dev)
        insts.append(Instance(samples=x, mpos=wl.mics.pos, gpos=wl.grid.pos, sample_freq=wl.fs,
                              block_size=wl.block_size, bin_lo=int(wl.bins[0]), num_bins=len(wl.bins),
                              precision='complex64'))
    plan = BatchPlan(insts, tc_precision=precision).capture()
    for _ in range(max(3, warmup)):
        plan.run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        e0.record()
        for _ in range(steps):
            plan.run()
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    units = plan.units()
    errs = {}
    for i in (0, len(wls) // 2, len(wls) - 1):
        mi = plan.map_instances[i]
        ref = D.map_f64(mi.csm, mi.wavenumbers, mi.mpos, mi.gpos, mi.steer_type, mi.r_diag, mi.norm,
                        clip_negative=mi.clip_negative)
        errs[f'inst{i}'] = dict(_err_vs(plan.out[i].cpu().numpy(), ref.cpu().numpy()), mics=int(wls[i].mics.num_mics),
                                grid_points=int(wls[i].grid.size))
    worst = {k: max(e[k] for e in errs.values()) for k in ('max_rel_err', 'rms_rel_err', 'peak_level_err_db')}
    mics = sorted({int(w.mics.num_mics) for w in wls})
    return {'value': units / (ms / 1e3), 'unit': UNIT, 'ms_per_step': ms, 'steps': steps, 'units_per_step': units,
            'config': {'workload': 'batched64', 'instances': len(wls), 'mics': mics,
                       'grid_points_range': [int(min(w.grid.size for w in wls)), int(max(w.grid.size for w in wls))],
                       'block_sizes': sorted({int(w.block_size) for w in wls}), 'bins_per_instance': 30,
                       'csm': 'complex64', 'form': f'tc {precision}', 'steer_type': 'true level', 'r_diag': True},
            'accuracy': {'vs': 'plain FP64 form on the same CSMs', **worst, 'instances': errs},
            'gpu_launches_per_step': '1 graph (per instance: FFT, Welch Gram, finalize; 1 batched map)',
            'clocks': clk.summary(), 'dtype': f'{precision} / f32 accum'}


def run_batched(args):
    d = batched_block(args.steps, args.warmup, args.tc_precision)
    _line('batched maps grid-pts*bins/s (64 uneven instances, CSM + map, one CUDA graph)', d['value'], UNIT,
          d['ms_per_step'], args, d['config'], units_per_step=d['units_per_step'], accuracy=d['accuracy'],
          gpu_launches_per_step=d['gpu_launches_per_step'], clocks=d['clocks'], dtype=d['dtype'])


def large3d_block(steps, warmup, precision):
    """1024-mic log spiral, 101x101x41 grid, 200 bins in 1-16 kHz, true location, r_diag.

    The CSM of the 200 bins is computed once (in contiguous bin chunks, then gathered); the timed step
    is the tensor-core map over all 200 bins and 418,241 grid points.  Accuracy and the FP64 form's rate
    on 3 bins.
    """
    import torch

    from acoular_b200 import device as D
    from acoular_b200 import workloads
    dev = torch.device('cuda', 0)
    wl = workloads.large_3d()
    M, G, N = wl.mics.num_mics, wl.grid.size, wl.block_size
    bins = np.asarray(wl.bins)
    nb = len(bins)
    x = workloads.monopole_time_data_torch(wl, device=dev)
    freqs = np.abs(np.fft.fftfreq(N, 1 / wl.fs)[: N // 2 + 1])
    mpos, gpos = torch.as_tensor(wl.mics.pos, device=dev), torch.as_tensor(wl.grid.pos, device=dev)
    k = torch.as_tensor(2 * np.pi * freqs[bins] / wl.c, device=dev)
    c = torch.empty((nb, M, M), dtype=torch.complex128, device=dev)
    t0 = time.perf_counter()
    for j0 in range(0, nb, 40):
        sel = bins[j0:j0 + 40]
        part = D.calc_csm(x, N, wl.window, wl.overlap, 'complex128', bin_lo=int(sel[0]),
                          num_bins=int(sel[-1] - sel[0] + 1))
        c[j0:j0 + len(sel)] = part[torch.as_tensor(sel - sel[0], device=dev)]
        del part
    torch.cuda.synchronize()
    csm_s = time.perf_counter() - t0
    del x
    out = torch.empty((nb, G), dtype=torch.float64, device=dev)
    norm = M / (M - 1.0)

    def step():
        D.map_tc(c, k, mpos, gpos, 'true location', True, norm, out=out, precision=precision)

    for _ in range(max(3, warmup)):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        e0.record()
        for _ in range(steps):
            step()
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    sel = torch.as_tensor([0, nb // 2, nb - 1], device=dev)
    cs, ks = c[sel].contiguous(), k[sel].contiguous()
    D.map_f64(cs, ks, mpos, gpos, 'true location', True, norm)
    torch.cuda.synchronize()
    e0.record()
    ref = D.map_f64(cs, ks, mpos, gpos, 'true location', True, norm)
    e1.record()
    torch.cuda.synchronize()
    f64_rate = 3 * G / (e0.elapsed_time(e1) / 1e3)
    rate = G * nb / (ms / 1e3)
    del c
    return {'value': rate, 'unit': UNIT, 'ms_per_step': ms, 'steps': steps,
            'config': {'workload': wl.name, 'mics': M, 'grid_points': G, 'bins': nb, 'block_size': N,
                       'steer_type': 'true location', 'r_diag': True, 'form': f'tc {precision}',
                       'csm': 'complex128, computed once outside the timed map steps'},
            'accuracy': {'vs': 'plain FP64 form', 'bins': [int(bins[0]), int(bins[nb // 2]), int(bins[-1])],
                         **_err_vs(out[sel].cpu().numpy(), ref.cpu().numpy())},
            'f64_form_rate': f64_rate, 'tc_over_f64': rate / f64_rate, 'csm_seconds_once': csm_s,
            'clocks': clk.summary(), 'dtype': f'{precision} / f32 accum'}


def run_large3d(args):
    d = large3d_block(args.steps, args.warmup, args.tc_precision)
    _line('map grid-pts*bins/s (1024 mics, 101x101x41 grid, 200 bins)', d['value'], UNIT, d['ms_per_step'], args,
          d['config'], accuracy=d['accuracy'], f64_form_rate=d['f64_form_rate'], tc_over_f64=d['tc_over_f64'],
          csm_seconds_once=d['csm_seconds_once'], clocks=d['clocks'], dtype=d['dtype'])


def serving_block(mixed: bool, duration: float, precision: str, verbose: bool = False):
    """Poisson arrivals from 32 streams, 0.1 s of 51.2 kHz samples per request, one third-octave band."""
    import torch

    from acoular_b200.microphones import disk_mics
    from acoular_b200.serving import BeamformingServer
    rng = np.random.RandomState(7)
    n_streams = 32
    srv = BeamformingServer(hbm_budget_bytes=120 << 30, tc_precision=precision)
    specs = []
    for i in range(n_streams):
        M = int(rng.choice([64, 128, 256, 512])) if mixed else 64
        side = int(rng.randint(41, 202))
        z = float(rng.uniform(-2.0, -0.3))
        g = np.linspace(-1.0, 1.0, side)
        gx, gy = np.meshgrid(g, g, indexing='ij')
        gpos = np.vstack([gx.ravel(), gy.ravel(), np.full(side * side, z)])
        N = int(rng.choice([256, 512, 1024]))
        while True:   # a third-octave band in 0.5-16 kHz that holds at least one FFT line
            fc = float(np.exp(rng.uniform(np.log(500.0), np.log(16000.0))))
            fr = np.abs(np.fft.fftfreq(N, 1 / 51200.0)[: N // 2 + 1])
            if np.searchsorted(fr, fc * 2 ** (-1 / 6)) < np.searchsorted(fr, fc * 2 ** (1 / 6)):
                break
        mpos = disk_mics(M, 0.5, seed=1000 + i).pos
        srv.open_stream(i, mpos, gpos, 51200.0, N, (fc, 3), gshape=(side, side))
        specs.append((M, side, N, fc))
    blocks = {i: rng.randn(5120, specs[i][0]).astype(np.float32) for i in range(n_streams)}
    # warm-up: one request per stream
    for f in [srv.submit(i, blocks[i]) for i in range(n_streams)]:
        f.result(timeout=120)
    torch.cuda.synchronize()
    rate = 10.0 * n_streams            # real time: each stream sends 0.1 s of data every 0.1 s
    futs = []
    with ClockSampler(0) as clk:
        # the arrival schedule starts once the clock sampler is up: arrivals due while it started would
        # otherwise be submitted together, as a burst that the offered load does not contain
        t_start = time.perf_counter()
        t_end = t_start + duration
        t_next = t_start
        while t_next < t_end:
            t_next += rng.exponential(1.0 / rate)
            delay = t_next - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            sid = int(rng.randint(n_streams))
            futs.append(srv.submit(sid, blocks[sid]))
        for f in futs:
            f.result(timeout=120)
        t_done = time.perf_counter()
    srv.close()
    lat = np.array([f.latency for f in futs]) * 1e3
    units = sum(f.units for f in futs) if all(hasattr(f, 'units') for f in futs) else None
    if verbose and srv.batch_times:
        bt = np.array(srv.batch_times)
        dur = (bt[:, 4] - bt[:, 1]) * 1e3
        top = np.argsort(dur)[-5:][::-1]
        print('slowest batches (n, inputs+csm issue ms, map issue ms, gpu wait ms):',
              [(int(bt[i, 0]), round((bt[i, 2] - bt[i, 1]) * 1e3, 2), round((bt[i, 3] - bt[i, 2]) * 1e3, 2),
                round((bt[i, 4] - bt[i, 3]) * 1e3, 2)) for i in top], file=sys.stderr)
    return {'p50_ms': float(np.percentile(lat, 50)), 'p99_ms': float(np.percentile(lat, 99)),
            'max_ms': float(lat.max()), 'requests': len(futs),
            'throughput_req_s': len(futs) / (t_done - t_start),
            'throughput_grid_pts_bins_s': (units / (t_done - t_start)) if units else None,
            'mean_batch': float(np.mean(srv.batches)) if srv.batches else None,
            'config': {'workload': 'serving-mixed' if mixed else 'serving-64mic', 'streams': n_streams,
                       'mics': sorted({s_[0] for s_ in specs}),
                       'grid_sides': [min(s_[1] for s_ in specs), max(s_[1] for s_ in specs)],
                       'block_sizes': sorted({s_[2] for s_ in specs}), 'offered_rate_req_s': rate,
                       'duration_s': duration, 'arrivals': 'Poisson', 'hbm_budget_gb': 120},
            'latency': 'wall clock from submit() to the host result, per request',
            'clocks': clk.summary(), 'dtype': f'{precision} / f32 accum'}


def run_serving(args, mixed: bool):
    d = serving_block(mixed, args.duration, args.tc_precision, verbose=True)
    _line('serving latency p50/p99 ms (Poisson arrivals, 32 streams, 0.1 s requests, one third-octave band)',
          d['p99_ms'], 'ms (p99)', d['p50_ms'], args, d['config'], higher_is_better=False, p50_ms=d['p50_ms'],
          p99_ms=d['p99_ms'], max_ms=d['max_ms'], requests=d['requests'], throughput_req_s=d['throughput_req_s'],
          throughput_grid_pts_bins_s=d['throughput_grid_pts_bins_s'], mean_batch=d['mean_batch'],
          clocks=d['clocks'], dtype=d['dtype'])


STEER_TYPES = ('classic', 'inverse', 'true level', 'true location')


def precision_matrix_block(csm64, kvec, mpos, gpos, acc_bins):
    """Every steering type x r_diag x tensor-core precision on the 256-mic workload's FP64 CSM (all bins,
    timed), each against the plain FP64 form on the bins ``acc_bins`` (errors) -- the map-only error of
    each tensor-core form -- and the rate ratio of the two forms (``tc_over_f64``)."""
    import torch

    from acoular_b200 import device as D
    dev = csm64.device
    nb, M, _ = csm64.shape
    G = gpos.shape[1]
    sel = torch.as_tensor(acc_bins, device=dev)
    cs, ks = csm64[sel].contiguous(), kvec[sel].contiguous()
    o = torch.empty((nb, G), dtype=torch.float64, device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        ev[0].record()
        r = fn()
        ev[1].record()
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]), r

    entries = {}
    for st in STEER_TYPES:
        for rd in (True, False):
            norm = M / (M - 1.0) if rd else 1.0
            f64_ms, ref = timed(lambda: D.map_f64(cs, ks, mpos, gpos, st, rd, norm))
            ref = ref.cpu().numpy()
            f64_rate = len(acc_bins) * G / (f64_ms / 1e3)
            for pr in ('tf32', 'bf16x3', 'fp16'):
                tc_ms, _ = timed(lambda: D.map_tc(csm64, kvec, mpos, gpos, st, rd, norm, out=o, precision=pr))
                rate = nb * G / (tc_ms / 1e3)
                entries[f'{st}|r_diag={rd}|{pr}'] = dict(_err_vs(o[sel].cpu().numpy(), ref), tc_rate=rate,
                                                         f64_rate=f64_rate, tc_over_f64=rate / f64_rate)
    worst = {k: max(e[k] for e in entries.values()) for k in ('max_rel_err', 'rms_rel_err', 'peak_level_err_db')}
    return {'vs': 'plain FP64 form (FP64 phase, libm-faithful float32 cos/sin) on the same FP64 CSM',
            'bins': [int(b) for b in acc_bins], 'worst': worst,
            'min_tc_over_f64': min(e['tc_over_f64'] for e in entries.values()),
            'definition': 'max/rms of |tc - f64| / max|f64| per bin over the listed bins; L_p difference at the '
                          'FP64 peak; tc_rate over all bins, f64_rate over the listed bins',
            'entries': entries}


def config1_block(steps, warmup):
    """The 64-mic, 41x41 workload (three monopoles, 51,200 samples, block 128, Hanning, 50 %): the full
    complex128 CSM (65 bins, 799 windows) and the plain FP64 map of the 8 kHz third-octave band (5 bins,
    'true level', r_diag) summed as BeamformerBase.synthetic sums it.  Device-timed with the samples
    resident, end to end through PowerSpectra + BeamformerBase.synthetic from host samples, and the CPU
    oracle on all host threads; the device band map against the oracle's."""
    import torch

    import acoular_b200 as ac
    from acoular_b200 import device as D
    from acoular_b200 import workloads
    from oracle import oracle as O
    dev = torch.device('cuda', 0)
    wl = workloads.three_sources_64()
    data = wl.time_data()
    M, G, N = wl.mics.num_mics, wl.grid.size, wl.block_size
    F = N // 2 + 1
    freqs = np.abs(np.fft.fftfreq(N, 1 / wl.fs)[:F])
    bins = np.arange(int(np.searchsorted(freqs, 8000.0 * 2.0 ** (-0.5 / 3))),
                     int(np.searchsorted(freqs, 8000.0 * 2.0 ** (0.5 / 3))))
    x = torch.as_tensor(data, device=dev)
    mpos, gpos = torch.as_tensor(wl.mics.pos, device=dev), torch.as_tensor(wl.grid.pos, device=dev)
    bsel = torch.as_tensor(bins, device=dev)
    kb = torch.as_tensor(2 * np.pi * freqs[bins] / wl.c, device=dev)
    norm = M / (M - 1.0)

    def step():
        csm = D.calc_csm(x, N, 'Hanning', '50%', 'complex128')
        return D.map_f64(csm[bsel].contiguous(), kb, mpos, gpos, 'true level', True, norm, clip_negative=True).sum(0)

    for _ in range(max(3, warmup)):
        band = step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        band = step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    got = band.cpu().numpy()
    e2e = []
    for it in range(4):
        t0 = time.perf_counter()
        ps = ac.PowerSpectra(source=ac.TimeSamples(data=data, sample_freq=wl.fs), block_size=N, window='Hanning',
                             overlap='50%')
        bf = ac.BeamformerBase(freq_data=ps, steer=ac.SteeringVector(grid=wl.grid, mics=wl.mics,
                                                                     steer_type='true level'), r_diag=True)
        syn = bf.synthetic(8000.0, 3)
        if it:
            e2e.append(time.perf_counter() - t0)
    O.set_num_threads(len(os.sched_getaffinity(0)))
    r0, rm = O.apparent_r(wl.grid.pos), O.apparent_r(wl.grid.pos, wl.mics.pos)
    cpu = []
    for it in range(3):
        t0 = time.perf_counter()
        c_ref = O.calc_csm(data, N, 'Hanning', '50%', 'complex128')
        ref = O.beamformer_calc(c_ref, freqs, bins, r0, rm, wl.c, 'true level', True)[bins].sum(0)
        if it:
            cpu.append(time.perf_counter() - t0)
    units = G * len(bins)
    err = float(np.abs(got - ref).max() / np.abs(ref).max())
    err_e2e = float(np.abs(np.asarray(syn).ravel() - ref).max() / np.abs(ref).max())
    return {'value': units / (ms / 1e3), 'unit': UNIT, 'ms_per_step': ms, 'steps': steps,
            'config': {'workload': wl.name, 'mics': M, 'grid_points': G, 'csm_bins': F, 'map_bins': [int(b) for b in bins],
                       'block_size': N, 'windows': D.num_windows(wl.num_samples, N, 2), 'steer_type': 'true level',
                       'r_diag': True, 'form': 'f64', 'csm': 'complex128'},
            'e2e': {'value': units / float(np.median(e2e)), 'unit': UNIT, 'ms': float(np.median(e2e)) * 1e3,
                    'h2d_bytes_per_step': int(data.nbytes), 'd2h_bytes_per_step': int(G * 8),
                    'api': 'TimeSamples -> PowerSpectra -> BeamformerBase.synthetic(8000, 3)'},
            'cpu_baseline': {'value': units / float(np.median(cpu)), 'unit': UNIT, 'ms': float(np.median(cpu)) * 1e3,
                             'cores': O.num_threads(), 'kind': 'port',
                             'sample': 'the whole step: CSM of 799 windows x 65 bins + the 5-bin band map'},
            'accuracy': {'vs': 'oracle', 'max_rel_err': err, 'e2e_max_rel_err': err_e2e},
            'gpu_launches_per_step': 4, 'dtype': 'f64'}


def run_eig(args):
    """Eigenvalue beamformer (BeamformerEig, n = -1) on the 256-mic workload: per step the largest eigenpair of
    all 513 CSMs (acb_heevd_select_f64, the path BeamformerEig takes for n = -1) and its map (plain FP64 form).
    The full decomposition (acb_heevd_f64) is timed beside it.  The CSM is computed once; the oracle checks 2
    bins."""
    import torch

    from acoular_b200 import device as D
    from acoular_b200 import workloads
    from oracle import oracle as O
    dev = torch.device('cuda', 0)
    wl = workloads.precision_256()
    M, G, N = wl.mics.num_mics, wl.grid.size, wl.block_size
    F = N // 2 + 1
    x = workloads.monopole_time_data_torch(wl, device=dev)
    csm = D.calc_csm(x, N, 'Hanning', '50%', 'complex128')
    del x
    if args.bins:   # profiling: the first bins only
        F = min(F, args.bins)
        csm = csm[:F].contiguous()
    freqs = np.abs(np.fft.fftfreq(N, 1 / wl.fs)[:F])
    k = torch.as_tensor(2 * np.pi * freqs / wl.c, device=dev)
    mpos, gpos = torch.as_tensor(wl.mics.pos, device=dev), torch.as_tensor(wl.grid.pos, device=dev)
    ev = torch.empty((F, 1), dtype=torch.float64, device=dev)
    evec = torch.empty((F, M, 1), dtype=torch.complex128, device=dev)
    out = torch.empty((F, G), dtype=torch.float64, device=dev)
    norm = M / (M - 1.0)
    ev_ms, map_ms = [], []
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]

    def step(rec=False):
        if rec:
            e[0].record()
        w_, v_ = D.heevd_select_f64(csm, [M - 1])
        ev.copy_(w_)
        evec.copy_(v_)
        if rec:
            e[1].record()
        D.map_eig_f64(ev, evec, k, mpos, gpos, 'true level', True, norm, clip_negative=True, out=out)
        if rec:
            e[2].record()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        t0.record()
        for _ in range(args.steps):
            step(rec=True)
            e[2].synchronize()
            ev_ms.append(e[0].elapsed_time(e[1]))
            map_ms.append(e[1].elapsed_time(e[2]))
        t1.record()
        torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / args.steps
    # the full decomposition (all eigenvectors, PowerSpectra.evd_device), outside the timed steps
    D.heevd_f64(csm)
    t0.record()
    w_full, _, _ = D.heevd_f64(csm)
    t1.record()
    torch.cuda.synchronize()
    full_ms = t0.elapsed_time(t1)
    top_err = float((w_full[:, M - 1] - ev[:, 0]).abs().max() / w_full[:, M - 1].abs().max())
    # end to end against the oracle (numpy eigh + the reference's eigen kernel) on 2 bins
    r0, rm = O.apparent_r(wl.grid.pos), O.apparent_r(wl.grid.pos, wl.mics.pos)
    errs = []
    check_bins = [b for b in (100, 400) if b < F] or [F - 1]
    for b in check_bins:
        c_h = csm[b].cpu().numpy()
        w, v = np.linalg.eigh(c_h)
        ref = O.beamformer_freq_eig('true level', True, norm, r0, rm, 2 * np.pi * freqs[b] / wl.c, w[M - 1:],
                                    np.ascontiguousarray(v[:, M - 1:]))[0]
        ref[ref < 0] = 0.0
        errs.append(float(np.abs(out[b].cpu().numpy() - ref).max() / np.abs(ref).max()))
    flops = 8.0 * M * G * F   # algorithmic: one complex M-vector product per grid-pt x bin
    _line('eigenvalue beamformer grid-pts*bins/s (BeamformerEig n=-1, 256 mics, 401x401 grid, 513 bins)',
          G * F / (ms / 1e3), UNIT, ms, args,
          {'workload': 'eig_' + wl.name, 'mics': M, 'grid_points': G, 'bins': F, 'components': 1,
           'steer_type': 'true level', 'r_diag': True, 'form': 'f64 (glibc-faithful steering)',
           'csm': 'complex128, computed once'},
          eigh_ms_per_step=float(np.mean(ev_ms)), full_eigh_ms=full_ms, top_eigval_vs_full=top_err,
          map_ms_per_step=float(np.mean(map_ms)),
          map_rate=G * F / (float(np.mean(map_ms)) / 1e3), map_tflops_algorithmic=flops / (np.mean(map_ms) / 1e3) / 1e12,
          accuracy={'vs': 'oracle (numpy eigh + the reference eigen kernel restated)', 'bins': check_bins,
                    'max_rel_err': max(errs)},
          gpu_launches_per_step='largest eigenpair (heevd_tridiag, heevd_select, heevd_back kernels) + 1 map_eig_small_kernel',
          clocks=clk.summary(),
          dtype='f64')


def run_damas(args):
    """DAMAS (BeamformerDamas defaults: true level, r_diag, n_iter 100, damp 1.0) on the 64-mic, 41x41
    workload's 8 kHz third-octave band (5 bins): per step the conventional maps, the 5 full PSFs
    (1681 x 1681) and the Gauss-Seidel solution.  The CSM is computed once; the oracle checks 1 bin."""
    import time

    import torch

    import acoular_b200 as ac
    from acoular_b200 import device as D
    from acoular_b200 import workloads
    from oracle import oracle as O
    dev = torch.device('cuda', 0)
    wl = workloads.three_sources_64()
    M, G, N = wl.mics.num_mics, wl.grid.size, wl.block_size
    F = N // 2 + 1
    x = workloads.monopole_time_data_torch(wl, device=dev)
    csm = D.calc_csm(x, N, 'Hanning', '50%', 'complex128')
    del x
    freqs = np.abs(np.fft.fftfreq(N, 1 / wl.fs)[:F])
    # the 8 kHz third-octave band as BeamformerBase.synthetic selects it
    bins = np.arange(int(np.searchsorted(freqs, 8000.0 * 2.0 ** (-0.5 / 3))),
                     int(np.searchsorted(freqs, 8000.0 * 2.0 ** (0.5 / 3))))
    B = bins.size
    n_iter, relax, st = 100, 1.0, 'true level'
    norm = M / (M - 1.0)
    mpos, gpos = torch.as_tensor(wl.mics.pos, device=dev), torch.as_tensor(wl.grid.pos, device=dev)
    steer = ac.SteeringVector(grid=wl.grid, mics=wl.mics, steer_type=st)
    r0_h, rm_h = np.ascontiguousarray(steer.r0), np.ascontiguousarray(steer.rm)
    r0, rm = torch.as_tensor(r0_h, device=dev), torch.as_tensor(rm_h, device=dev)
    csm_b = csm[torch.as_tensor(bins, device=dev)].contiguous()
    psf = torch.empty((B, G, G), dtype=torch.float64, device=dev)
    src = torch.arange(G, device=dev)
    sol = torch.empty((B, G), dtype=torch.float64, device=dev)
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    st_ms = {'map': [], 'psf': [], 'gauss_seidel': []}

    kb_h = 2 * np.pi * freqs[bins] / wl.c
    kb = [float(v) for v in kb_h]
    kb_t = torch.as_tensor(kb_h, device=dev)

    def step(rec=False):   # wave numbers as host floats: no synchronisation inside the step
        if rec:
            e[0].record()
        y = D.map_f64(csm_b, kb_t, mpos, gpos, st, True, norm, clip_negative=True)
        if rec:
            e[1].record()
        for j in range(B):
            D.psf_f64(r0, rm, kb[j], src, st, out=psf[j])
        if rec:
            e[2].record()
        sol.copy_(y)
        D.damas_gauss_seidel(psf, y, n_iter, relax, solution=sol)
        if rec:
            e[3].record()

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        t0.record()
        for _ in range(args.steps):
            step(rec=True)
            e[3].synchronize()
            st_ms['map'].append(e[0].elapsed_time(e[1]))
            st_ms['psf'].append(e[1].elapsed_time(e[2]))
            st_ms['gauss_seidel'].append(e[2].elapsed_time(e[3]))
        t1.record()
        torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / args.steps
    # accuracy: one bin against the oracle (the reference's PSF and Gauss-Seidel restated)
    b0 = int(bins[B // 2])
    c_h = csm[b0:b0 + 1].cpu().numpy()
    tc = time.perf_counter()
    ref = O.beamformer_damas_calc(c_h, freqs[b0:b0 + 1], [0], r0_h, rm_h, wl.c, st, True, n_iter, relax)[0]
    cpu_s = time.perf_counter() - tc
    got = sol[B // 2].cpu().numpy()
    err = float(np.abs(got - ref).max() / np.abs(ref).max())
    # end to end through the public API: host CSM -> PowerSpectraImport -> BeamformerDamas -> band map
    c_host = csm.cpu().numpy()
    e2e_ms = []
    for it in range(max(2, min(args.steps, 5)) + 1):
        torch.cuda.synchronize()
        ta = time.perf_counter()
        ps = ac.PowerSpectraImport(csm=c_host, frequencies=freqs)
        bf = ac.BeamformerDamas(freq_data=ps, steer=steer, r_diag=True, n_iter=n_iter, damp=relax)
        band = np.asarray(bf.result[int(bins[0]):int(bins[-1]) + 1])
        if it:
            e2e_ms.append((time.perf_counter() - ta) * 1e3)
    e2e_err = float(np.abs(band[B // 2] - ref).max() / np.abs(ref).max())
    gs_ms = float(np.mean(st_ms['gauss_seidel']))
    pk = peaks()
    gs_bytes = float(B) * n_iter * G * G * 8.0       # the PSF read once per sweep
    achieved = gs_bytes / (gs_ms / 1e3) / 1e9
    nblk = (G + 31) // 32
    _line('DAMAS bins/s (BeamformerDamas, 64 mics, 41x41 grid, 8 kHz third-octave band, n_iter 100)',
          B / (ms / 1e3), 'bins/s', ms, args,
          {'workload': 'damas_' + wl.name, 'mics': M, 'grid_points': G, 'bins': B, 'n_iter': n_iter, 'damp': relax,
           'steer_type': st, 'r_diag': True, 'psf': 'full (G x G per bin), float64',
           'csm': 'complex128, computed once', 'l2': 'psf of the band (113 MB) read 100x per step'},
          stage_ms={k: float(np.mean(v)) for k, v in st_ms.items()},
          roofline={'kernel': 'damas_kernel', 'bound': 'hbm (latency: one 32-row block per step)',
                    'achieved': achieved, 'peak': pk['hbm_gbs'], 'unit': 'GB/s', 'frac': achieved / pk['hbm_gbs'],
                    'traffic': None, 'bytes_per_launch': gs_bytes,
                    'sequential_steps_per_launch': n_iter * nblk,
                    'us_per_step': gs_ms * 1e3 / (n_iter * nblk)},
          psf_rate_elems_per_s=B * G * G * M / (float(np.mean(st_ms['psf'])) / 1e3),
          accuracy={'vs': 'oracle (the reference PSF and Gauss-Seidel restated)', 'bin': b0, 'max_rel_err': err,
                    'e2e_max_rel_err': e2e_err},
          e2e={'value': B / (float(np.median(e2e_ms)) / 1e3), 'unit': 'bins/s',
               'ms': float(np.median(e2e_ms)),
               'h2d_bytes_per_step': int(c_host.nbytes + r0_h.nbytes + rm_h.nbytes + 2 * 3 * 8 * (G + M)),
               'd2h_bytes_per_step': int(B * G * 8)},
          cpu_baseline={'value': 1.0 / cpu_s, 'unit': 'bins/s', 'cores': O.num_threads(), 'kind': 'port',
                        'sample': f'1 bin (bin {b0}): map + full PSF + {n_iter} sweeps'},
          gpu_launches=f'{1 + B + 1} per step (map_plain_kernel, {B} psf_kernel, damas_kernel) + 1 copy',
          clocks=clk.summary(), dtype='f64')


def run_cleansc(args):
    """CLEAN-SC (BeamformerCleansc defaults: true level, r_diag, n_iter 0 = up to 2 M = 128 iterations,
    damp 0.6, stopn 3) on the 64-mic, 41x41 workload's 8 kHz third-octave band (5 bins): per step the
    conventional maps and every iteration of all 5 bins.  The CSM is computed once; the oracle checks 1 bin."""
    import time

    import torch

    import acoular_b200 as ac
    from acoular_b200 import device as D
    from acoular_b200 import workloads
    from oracle import oracle as O
    dev = torch.device('cuda', 0)
    wl = workloads.three_sources_64()
    M, G, N = wl.mics.num_mics, wl.grid.size, wl.block_size
    F = N // 2 + 1
    x = workloads.monopole_time_data_torch(wl, device=dev)
    csm = D.calc_csm(x, N, 'Hanning', '50%', 'complex128')
    del x
    freqs = np.abs(np.fft.fftfreq(N, 1 / wl.fs)[:F])
    bins = np.arange(int(np.searchsorted(freqs, 8000.0 * 2.0 ** (-0.5 / 3))),
                     int(np.searchsorted(freqs, 8000.0 * 2.0 ** (0.5 / 3))))
    B = bins.size
    st, n_iter, damp, stopn = 'true level', 0, 0.6, 3
    norm = M / (M - 1.0)
    mpos, gpos = torch.as_tensor(wl.mics.pos, device=dev), torch.as_tensor(wl.grid.pos, device=dev)
    csm_b = csm[torch.as_tensor(bins, device=dev)].contiguous()
    kb = torch.as_tensor(2 * np.pi * freqs[bins] / wl.c, device=dev)

    def step():
        return D.cleansc_f64(csm_b, kb, st, True, norm, n_iter, damp, stopn, mpos=mpos, gpos=gpos)

    for _ in range(max(3, args.warmup)):
        res = step()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        t0.record()
        for _ in range(args.steps):
            res = step()
        t1.record()
        torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / args.steps
    steer = ac.SteeringVector(grid=wl.grid, mics=wl.mics, steer_type=st)
    r0_h, rm_h = np.ascontiguousarray(steer.r0), np.ascontiguousarray(steer.rm)
    b0 = int(bins[B // 2])
    c_h = csm[b0:b0 + 1].cpu().numpy()
    tc = time.perf_counter()
    ref = O.beamformer_cleansc_calc(c_h, freqs[b0:b0 + 1], [0], r0_h, rm_h, wl.c, st, True, n_iter, damp, stopn)[0]
    cpu_s = time.perf_counter() - tc
    got = res[B // 2].double().cpu().numpy()
    err = float(np.abs(got - ref).max() / np.abs(ref).max())
    same_peaks = bool(np.array_equal(got != 0, ref != 0))
    c_host = csm.cpu().numpy()
    e2e_ms = []
    for it in range(max(2, min(args.steps, 5)) + 1):
        torch.cuda.synchronize()
        ta = time.perf_counter()
        ps = ac.PowerSpectraImport(csm=c_host, frequencies=freqs)
        bf = ac.BeamformerCleansc(freq_data=ps, steer=steer, r_diag=True, n_iter=n_iter, damp=damp, stopn=stopn)
        band = np.asarray(bf.result[int(bins[0]):int(bins[-1]) + 1])
        if it:
            e2e_ms.append((time.perf_counter() - ta) * 1e3)
    e2e_err = float(np.abs(band[B // 2] - ref).max() / np.abs(ref).max())
    J = 2 * M
    _line('CLEAN-SC bins/s (BeamformerCleansc, 64 mics, 41x41 grid, 8 kHz third-octave band)', B / (ms / 1e3),
          'bins/s', ms, args,
          {'workload': 'cleansc_' + wl.name, 'mics': M, 'grid_points': G, 'bins': B, 'n_iter': 'auto (<= 128)',
           'damp': damp, 'stopn': stopn, 'steer_type': st, 'r_diag': True, 'csm': 'complex128, computed once'},
          accuracy={'vs': 'oracle (the reference CLEAN-SC restated)', 'bin': b0, 'max_rel_err': err,
                    'same_peaks': same_peaks, 'e2e_max_rel_err': e2e_err},
          e2e={'value': B / (float(np.median(e2e_ms)) / 1e3), 'unit': 'bins/s', 'ms': float(np.median(e2e_ms)),
               'h2d_bytes_per_step': int(c_host.nbytes + r0_h.nbytes + rm_h.nbytes),
               'd2h_bytes_per_step': int(B * G * 4)},
          cpu_baseline={'value': 1.0 / cpu_s, 'unit': 'bins/s', 'cores': O.num_threads(), 'kind': 'port',
                        'sample': f'1 bin (bin {b0}): map + CLEAN-SC iterations'},
          gpu_launches=f'{2 + 2 * J - 1} per step (init, map_plain_kernel, {J} cleansc_step_kernel, '
                       f'{J - 1} map_eig_small_kernel; stopped bins return at once)',
          clocks=clk.summary(), dtype='f64')


def run_stream(args):
    """Streaming spectra (RFFT -> CrossPowerSpectra, calc_mode 'full', complex128) of the 64-mic
    workload's 1 s of samples (51,200 samples x 64 channels, block 128, Hanning, 50 %): per step every
    snapshot's 65 bins x 64 x 64 matrix, in device blocks of 64 snapshots (samples resident)."""
    import time

    import torch

    import acoular_b200 as ac
    from acoular_b200 import workloads
    from oracle import oracle as O
    dev = torch.device('cuda', 0)
    wl = workloads.three_sources_64()
    data = wl.time_data()
    ts_dev = ac.TimeSamples(data=torch.as_tensor(data, device=dev), sample_freq=wl.fs)
    N, M = 128, wl.mics.num_mics
    F = N // 2 + 1
    num = 64
    rf = ac.RFFT(source=ts_dev, block_size=N, window='Hanning', overlap='50%')
    cps = ac.CrossPowerSpectra(source=rf)
    K = (data.shape[0] - N) // (N // 2) + 1
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    sink = torch.zeros((F, M, M), dtype=torch.complex128, device=dev)

    def step():
        for b in cps.result_device(num):
            sink.add_(b[-1])      # consume each block on the device (its last snapshot)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    with ClockSampler(0) as clk:
        ev[0].record()
        for _ in range(args.steps):
            step()
        ev[1].record()
        torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[1]) / args.steps
    # the cross-spectra kernel alone on one block, for the roofline (bytes written + spectra read)
    spec = next(rf.result_device(num))
    from acoular_b200 import _native as NAT
    out = torch.empty((num, F, M, M), dtype=torch.complex128, device=dev)
    for _ in range(3):
        NAT.check(NAT.lib().acb_cross_spectra(spec.data_ptr(), num, F, M, NAT.C128, 1.0, out.data_ptr(),
                                              NAT.stream_handle()), 'acb_cross_spectra')
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 20
    e0.record()
    for _ in range(reps):
        NAT.check(NAT.lib().acb_cross_spectra(spec.data_ptr(), num, F, M, NAT.C128, 1.0, out.data_ptr(),
                                              NAT.stream_handle()), 'acb_cross_spectra')
    e1.record()
    torch.cuda.synchronize()
    k_ms = e0.elapsed_time(e1) / reps
    k_bytes = num * F * M * M * 16.0 + num * F * M * 16.0
    pk = peaks()
    achieved = k_bytes / (k_ms / 1e3) / 1e9
    # end to end from host samples: TimeSamples(numpy) -> RFFT -> CrossPowerSpectra.result (numpy blocks)
    ts_host = ac.TimeSamples(data=data, sample_freq=wl.fs)
    e2e = []
    for it in range(3):
        torch.cuda.synchronize()
        ta = time.perf_counter()
        n_out = 0
        for b in ac.CrossPowerSpectra(source=ac.RFFT(source=ts_host, block_size=N, window='Hanning',
                                                     overlap='50%')).result(num):
            n_out += b.shape[0]
        if it:
            e2e.append((time.perf_counter() - ta) * 1e3)
    # oracle on a bounded sample: 64 snapshots
    tc = time.perf_counter()
    blocks = list(O.rfft_blocks(data[: (num + 1) * N // 2], N, 'Hanning', '50%', 'complex128', 'none', num))
    ref = list(O.cross_power_blocks(blocks, F, M, O.power_scale(N, wl.fs, 'power', True), 'complex128'))
    cpu_s = time.perf_counter() - tc
    got = next(cps.result(num))
    err = float(np.abs(got - ref[0]).max() / np.abs(ref[0]).max())
    n_cpu = sum(b.shape[0] for b in ref)
    _line('streaming cross-spectra snapshots/s (RFFT -> CrossPowerSpectra full, 64 mics, block 128, 65 bins)',
          K / (ms / 1e3), 'snapshots/s', ms, args,
          {'workload': 'stream_' + wl.name, 'mics': M, 'block_size': N, 'window': 'Hanning', 'overlap': '50%',
           'snapshots': K, 'block_num': num, 'precision': 'complex128',
           'out_bytes_per_step': K * F * M * M * 16},
          roofline={'kernel': 'cross_spectra_kernel', 'bound': 'hbm', 'achieved': achieved, 'peak': pk['hbm_gbs'],
                    'unit': 'GB/s', 'frac': achieved / pk['hbm_gbs'], 'traffic': None, 'bytes_per_launch': k_bytes,
                    'ms_per_launch': k_ms},
          accuracy={'vs': 'oracle (the reference generators restated)', 'block': 0, 'max_rel_err': err},
          e2e={'value': n_out / (float(np.median(e2e)) / 1e3), 'unit': 'snapshots/s', 'ms': float(np.median(e2e)),
               'h2d_bytes_per_step': int(data.nbytes), 'd2h_bytes_per_step': int(n_out * F * M * M * 16)},
          cpu_baseline={'value': n_cpu / cpu_s, 'unit': 'snapshots/s', 'cores': O.num_threads(), 'kind': 'port',
                        'sample': f'{n_cpu} snapshots'},
          gpu_launches=f'{3 * -(-K // num)} per step (fft_window_kernel, spectra_pack_kernel, cross_spectra_kernel '
                       f'per block of {num}) + the consumer',
          clocks=clk.summary(), dtype='f64')


def main():
    args = parse()
    if args.workload == 'stream':
        return run_stream(args)
    if args.workload == 'cleansc':
        return run_cleansc(args)
    from acoular_b200 import workloads
    if args.workload == 'eig':
        return run_eig(args)
    if args.workload == 'damas':
        return run_damas(args)
    if args.workload == 'batched64':
        return run_batched(args)
    if args.workload == 'large3d':
        return run_large3d(args)
    if args.workload in ('serving', 'serving-mixed'):
        return run_serving(args, args.workload == 'serving-mixed')
    wl = workloads.precision_256()
    if args.impl == 'reference':
        return run_reference(args, wl)

    import torch

    from acoular_b200 import _native as NAT
    from acoular_b200 import device as D
    ws, rank, local = dist_setup(args)
    dev = torch.device('cuda', local)
    form = args.form or ('tc' if hasattr(D, 'map_tc') else 'f64')
    M, G, N = wl.mics.num_mics, wl.grid.size, wl.block_size
    F = N // 2 + 1
    nbins = args.bins or F
    bins = np.arange(F)[:nbins]

    # resident inputs
    samples = workloads.monopole_time_data_torch(wl, device=dev)
    mpos = torch.as_tensor(wl.mics.pos, device=dev)
    gpos = torch.as_tensor(wl.grid.pos, device=dev)
    freqs = np.abs(np.fft.fftfreq(N, 1 / wl.fs)[:F])
    kvec = torch.as_tensor(2 * np.pi * freqs[bins] / wl.c, device=dev)
    norm = M / (M - 1.0)
    out = torch.empty((nbins, G), dtype=torch.float64, device=dev)
    K = D.num_windows(wl.num_samples, N, 2)
    prec = args.tc_precision
    # the CSM in the same form as the map: FP64 Gram for the FP64 form, tensor-core Gram otherwise
    # the tensor-core CSM has TF32 and split-BF16 forms; the FP16 map takes the TF32 CSM
    csm_tc = 'tf32' if prec == 'fp16' else prec
    csm_prec = 'complex128' if form == 'f64' else f'tc_{csm_tc}'
    ws_bytes = NAT.lib().acb_csm_workspace_bytes(M, F, K, D.CSM_PRECISIONS[csm_prec])
    workspace = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    csm_up = torch.zeros((F, M, M), dtype=torch.complex128, device=dev)
    csm_full = torch.empty((F, M, M), dtype=torch.complex128, device=dev)
    _, weight = D.window_vector('Hanning', N, dev)
    scale = 2.0 / N / weight / D.num_blocks(wl.num_samples, N, 2)
    ev_map = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev_csm = torch.cuda.Event(enable_timing=True)
    map_ms, csm_ms = [], []

    def step(record=False):
        if record:
            ev_csm.record()
        csm_up.zero_()
        D.csm_upper_accumulate(samples, N, 'Hanning', '50%', precision=csm_prec, csm_upper=csm_up, workspace=workspace,
                               max_workspace_bytes=ws_bytes)
        D.csm_finalize(csm_up, scale, out=csm_full)
        c = csm_full if nbins == F else csm_full[:nbins]
        if record:
            ev_map[0].record()
        if form == 'f64':
            D.map_f64(c, kvec, mpos, gpos, args.steer, True, norm, out=out)
        else:
            D.map_tc(c, kvec, mpos, gpos, args.steer, True, norm, out=out, precision=prec)
        if record:
            ev_map[1].record()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record()
        for _ in range(args.steps):
            step(record=True)
            ev_map[1].synchronize()
            map_ms.append(ev_map[0].elapsed_time(ev_map[1]))
            csm_ms.append(ev_csm.elapsed_time(ev_map[0]))
        e1.record()
        torch.cuda.synchronize()
    barrier(ws)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    ms = max_over_ranks(ms, ws)
    units = float(G) * nbins
    value = units * ws / (ms / 1e3)

    # the forms side by side on the same CSM: both tensor-core precisions over all bins, and the plain
    # FP64 form on a spread of 6 bins (its rate per grid-pt x bin does not depend on the bin)
    acc_bins = np.unique(np.linspace(min(2, nbins - 1), nbins - 1, 6).round().astype(int))
    if acc_bins.min() < 0 or acc_bins.max() >= nbins:   # checked on the host, before any device indexing
        raise ValueError(f'accuracy bins {acc_bins.tolist()} outside the {nbins} map bins')
    sel = torch.as_tensor(acc_bins, device=dev)
    accuracy, forms = None, {}
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn, reps=2):
        fn()
        torch.cuda.synchronize()
        ev[0].record()
        for _ in range(reps):
            r = fn()
        ev[1].record()
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]) / reps, r

    c_all = csm_full if nbins == F else csm_full[:nbins]
    # reference: the FP64 CSM (the reference's arithmetic) and the plain FP64 map on it
    del workspace
    csm64 = c_all if csm_prec == 'complex128' else D.calc_csm(samples, N, 'Hanning', '50%', 'complex128')[:nbins]
    cs, ks = csm64[sel].contiguous(), kvec[sel].contiguous()
    f64_ms, ref_t = timed(lambda: D.map_f64(cs, ks, mpos, gpos, args.steer, True, norm), reps=1)
    ref_map = ref_t.cpu().numpy()
    forms['f64'] = {'rate': len(acc_bins) * G / (f64_ms / 1e3), 'bins_timed': len(acc_bins)}
    lp = lambda x: 10 * np.log10(np.maximum(x / 4e-10, np.finfo(np.float64).eps))  # noqa: E731

    def acc_of(m):
        got = m[sel].cpu().numpy()
        err = np.abs(got - ref_map) / np.abs(ref_map).max(axis=1, keepdims=True)
        peak = ref_map.argmax(axis=1)
        db = np.abs(lp(got[np.arange(len(acc_bins)), peak]) - lp(ref_map[np.arange(len(acc_bins)), peak]))
        return {'max_rel_err': float(err.max()), 'rms_rel_err': float(np.sqrt((err ** 2).mean())),
                'peak_level_err_db': float(db.max())}

    if form != 'f64':
        out2 = torch.empty_like(out)
        for pr in ('bf16x3', 'tf32', 'fp16'):
            o = out if pr == prec else out2
            t_ms, _ = timed(lambda: D.map_tc(c_all, kvec, mpos, gpos, args.steer, True, norm, out=o, precision=pr))
            forms[f'tc_{pr}'] = {'rate': units / (t_ms / 1e3), 'map_ms': t_ms, 'tc_over_f64':
                                 units / (t_ms / 1e3) / forms['f64']['rate'],
                                 'map_only_err': acc_of(D.map_tc(csm64, kvec, mpos, gpos, args.steer, True, norm,
                                                                 precision=pr))}
            if pr == prec:
                forms[f'tc_{pr}']['end_to_end_err'] = acc_of(o)
        accuracy = {'vs': 'FP64 CSM + plain FP64 map (the reference arithmetic on the GPU)',
                    'timed_path': f'{csm_prec} CSM + tc {prec} map', 'bins': acc_bins.tolist(), **acc_of(out),
                    'definition': '|map - ref| / max|ref| per bin; L_p difference at the reference peak'}
    pmatrix = None
    if form != 'f64' and not args.no_extra and rank == 0:
        pmatrix = precision_matrix_block(csm64, kvec, mpos, gpos, acc_bins)

    # map kernel roofline: algorithmic flops 8 M^2 + 8 M per grid-pt x bin
    pk = peaks()
    gp = gemm_peaks(dev)
    flops = (8.0 * M * M + 8.0 * M) * units
    map_avg = float(np.mean(map_ms))
    achieved_tf = flops / (map_avg / 1e3) / 1e12
    if form == 'f64':
        roof = {'bound': 'fp64', 'achieved': achieved_tf, 'peak': gp['fp64_tflops'], 'unit': 'TFLOP/s',
                'frac': achieved_tf / gp['fp64_tflops'], 'traffic': None, 'kernel': 'map_plain_kernel',
                'peak_kind': 'DGEMM measured in this run'}
    else:
        # denominator: the measured sustained BF16 rate of the peak file (dense FP16 runs at the BF16 rate,
        # dense TF32 at half of it, so for TF32 it is the conservative one; the cuBLAS TF32 GEMM measured
        # in this run is given beside it)
        steer_idx = STEER_TYPES.index(args.steer) + 1
        tpb = TC_TRAFFIC_PER_BIN.get(prec)
        roof = {'bound': 'tensor', 'achieved': achieved_tf, 'peak': pk['bf16_tflops_sustained'], 'unit': 'TFLOP/s',
                'frac': achieved_tf / pk['bf16_tflops_sustained'], 'traffic': None if tpb is None else tpb * nbins,
                'kernel': f'map_tc_kernel<{steer_idx},{TC_PREC_INDEX[prec]}>',
                'peak_kind': f"bf16 sustained ({pk['source']})"}
        if prec == 'tf32':
            roof['frac_of_tf32_gemm_here'] = achieved_tf / gp['tf32_tflops']
    if roof['traffic'] is not None:
        roof['traffic_note'] = ('DRAM bytes per launch: ncu dram__bytes_read+write of the whole 513-bin launch '
                                '(per-bin figure x bins); algorithmic bytes: the map written once plus each bin\'s R\' '
                                'tiles read once')

    # end to end through the public API (pinned host samples -> host result)
    e2e = None
    if not args.no_e2e:
        import acoular_b200 as ac
        host = torch.empty((wl.num_samples, M), dtype=torch.float32, pin_memory=True)
        host.copy_(samples.cpu())
        ts = ac.TimeSamples(data=host, sample_freq=wl.fs)
        times = []
        for i in range(2 + max(1, min(args.steps, 3))):
            ps = ac.PowerSpectra(source=ts, block_size=N, window='Hanning', overlap='50%',
                                 form='f64' if form == 'f64' else 'tc', tc_precision=csm_tc)
            st = ac.SteeringVector(grid=wl.grid, mics=wl.mics, steer_type=args.steer)
            bb = ac.BeamformerBase(freq_data=ps, steer=st, r_diag=True, form=form, tc_precision=prec)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = bb.result[0:nbins]
            t = time.perf_counter() - t0
            if i >= 2:
                times.append(t)
        e2e_s = max_over_ranks(float(np.median(times)), ws)
        e2e = {'value': units * ws / e2e_s, 'unit': UNIT, 'h2d_bytes_per_step': int(host.numel() * 4),
               'd2h_bytes_per_step': int(res.nbytes), 'ms_per_step': e2e_s * 1e3}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline_sample(wl, args.steer)

    # the other configurations, each timed on its own (rank 0 at N = 1): their rates, errors and latencies
    extra = {}
    if rank == 0 and ws == 1 and not args.no_extra:
        del samples, csm_up, csm_full, out, csm64, cs, ks
        torch.cuda.empty_cache()
        extra['config1'] = config1_block(20, 3)
        extra['batched64'] = batched_block(10, 3, prec)
        torch.cuda.empty_cache()
        extra['large3d'] = large3d_block(2, 3, prec)
        torch.cuda.empty_cache()
        extra['serving'] = serving_block(False, 5.0, prec)
        extra['serving_mixed'] = serving_block(True, 5.0, prec)

    if rank == 0:
        line = {'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': ws, 'steps': args.steps,
                'warmup': args.warmup, 'ms_per_step': ms, 'higher_is_better': True, 'scaling': 'weak',
                'vs_baseline': None,
                'dtype': 'f64' if form == 'f64' else TC_DTYPE[prec],
                'data': 'synthetic (seeded monopoles, GPU-generated)',
                'config': {'workload': wl.name, 'mics': M, 'grid_points': G, 'bins': nbins, 'block_size': N,
                           'windows': K, 'steer_type': args.steer, 'r_diag': True, 'form': form, 'csm': csm_prec,
                           'l2': 'inputs larger than L2 (samples 524 MB, CSM 538 MB, map 660 MB)',
                           'parallelism': f'{ws} independent instances (one per GPU)'},
                'map_ms_per_step': map_avg, 'csm_ms_per_step': float(np.mean(csm_ms)),
                'csm_rate': {'value': units / (float(np.mean(csm_ms)) / 1e3), 'unit': UNIT,
                             'note': f'CSM stage alone (FFT + {csm_prec} Welch Gram + finish), all bins'},
                'forms': forms, 'gemm_peaks_here': gp,
                'roofline': roof, 'accuracy': accuracy, 'cpu_baseline': cpu, 'e2e': e2e,
                'gpu_launches': None, 'clocks': clk.summary()}
        if pmatrix is not None:
            line['precision_matrix'] = pmatrix
        line.update(extra)
        line['gpu_launches'] = launches_per_step(F, nbins, K, M) * args.steps
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def launches_per_step(F, nbins, K, M):
    # csm_up.zero_ is a torch fill (not counted); ours: fft + gram per workspace chunk, finalize, map
    chunks = -(-K // 65535)
    return 2 * chunks + 1 + 1


if __name__ == '__main__':
    main()
