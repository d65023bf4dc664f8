"""Autotuner of the tensor-core map: accumulator tile width and split, per shape class.

The tensor-core map kernel (``acb_map_tc_batch``) has two free parameters per instance:

* ``pass_chunks`` -- the accumulator tile width: the columns of the block-triangular product are
  covered in passes of 4, 8 or 16 chunks (128, 256 or 512 TMEM columns).  Narrower passes leave
  room for more accumulator windows in TMEM (the next item's MMAs start while the epilogue still
  drains the previous one) but re-synthesise the steering chunks of every earlier pass.
* ``splits`` -- how many CTAs share one (bin, 128-point tile): its passes are cut into that many
  groups of balanced cost, each group's partial sums go to a workspace and the last group to
  finish combines them in group order.  Splits fill the SMs when a request has few tiles of a
  large array; they cost the partial-sum traffic and repeat the early steering chunks.

A *shape class* is (operand precision, padded mic count rounded up to a power of two, work-item
bucket): the item bucket is ``tiny`` (bins x tiles <= 37, a quarter of the SMs or less: the
class where a split can shorten the launch), ``few`` (<= 148, at most one item per SM), ``mid``
(<= 8 waves) or ``many``.  :func:`tune` times every candidate on a representative instance of
each class on the current GPU and writes the winners, with all measured times, to
``tuning/map_tc_b200.json``; :func:`lookup` reads that table (a class missing from it gets the
default: widest tile, no split).  The results of an instance depend only on its own shape class,
never on what shares its launch.

Run on a B200:  ``python -m acoular_b200.autotune [--out PATH] [--reps N]``.
"""

from __future__ import annotations

import json
import math
import time
from functools import lru_cache
from pathlib import Path

import numpy as np

TABLE_PATH = Path(__file__).resolve().parent / 'tuning' / 'map_tc_b200.json'
PASS_CHUNKS = (4, 8, 16)
SPLITS = (1, 2, 4, 8)
MIC_BUCKETS = (32, 64, 128, 256, 512, 1024, 2048)
NUM_SMS = 148
DEFAULT = (16, 1)

# representative (grid side, bins) per item bucket: 14 tiles x 2 bins, 14 x 8, 80 x 12, 316 x 16
REPRESENTATIVE = {'tiny': (41, 2), 'few': (41, 8), 'mid': (101, 12), 'many': (201, 16)}


def mic_bucket(num_mics: int) -> int:
    mp = (int(num_mics) + 15) // 16 * 16
    for b in MIC_BUCKETS:
        if mp <= b:
            return b
    return MIC_BUCKETS[-1]


def item_bucket(num_grid: int, num_bins: int) -> str:
    items = int(num_bins) * ((int(num_grid) + 127) // 128)
    if 4 * items <= NUM_SMS:
        return 'tiny'
    if items <= NUM_SMS:
        return 'few'
    if items <= 8 * NUM_SMS:
        return 'mid'
    return 'many'


def shape_class(num_mics: int, num_grid: int, num_bins: int, precision: str) -> str:
    return f'{precision}:m{mic_bucket(num_mics)}:{item_bucket(num_grid, num_bins)}'


def candidates(num_mics: int):
    """Distinct (pass_chunks, splits) for this mic count (same pass count = same schedule)."""
    C = (int(num_mics) + 15) // 16
    out, seen = [], set()
    for pw in PASS_CHUNKS:
        P = math.ceil(C / pw)
        for sp in SPLITS:
            if sp > P or (P, sp, min(C, pw)) in seen:
                continue
            seen.add((P, sp, min(C, pw)))
            out.append((pw, sp))
    return out


@lru_cache(maxsize=4)
def _load(path: str) -> dict:
    p = Path(path)
    if not p.exists():
        return {}
    return json.loads(p.read_text()).get('classes', {})


def lookup(num_mics: int, num_grid: int, num_bins: int, precision: str, path: Path | str = TABLE_PATH):
    """(pass_chunks, splits) for an instance: the tuned entry of its class, else the default."""
    ent = _load(str(path)).get(shape_class(num_mics, num_grid, num_bins, precision))
    if not ent:
        return DEFAULT
    pw, sp = int(ent['pass_chunks']), int(ent['splits'])
    C = (int(num_mics) + 15) // 16
    if pw not in PASS_CHUNKS or sp < 1 or sp > max(1, math.ceil(C / pw)):
        return DEFAULT
    return pw, sp


def _instance(M: int, side: int, nbins: int, dev, seed: int = 0):
    """A seeded Hermitian PSD CSM (64 random spectra per bin, made on the device) on a disk array,
    a square grid.  Timing does not depend on the CSM's values."""
    import torch

    from . import device as D
    from .microphones import disk_mics
    mpos = disk_mics(M, 0.5, seed=seed + 1).pos
    g = np.linspace(-0.5, 0.5, side)
    gx, gy = np.meshgrid(g, g, indexing='ij')
    gpos = np.vstack([gx.ravel(), gy.ravel(), np.full(side * side, -1.0)])
    gen = torch.Generator(device=dev).manual_seed(seed)
    X = torch.randn((nbins, 64, M), dtype=torch.complex128, device=dev, generator=gen)
    csm = (X.conj().transpose(1, 2) @ X / 64.0).contiguous()
    k = 2 * np.pi * np.linspace(1000.0, 12000.0, nbins) / 343.0
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)  # noqa: E731
    return D.MapInstance(csm, t(k), t(mpos), t(gpos), 'true level', True, M / (M - 1.0))


def _time(mi, precision: str, tuning, reps: int) -> float:
    import torch

    from . import device as D
    mi.tuning = tuning
    for _ in range(2):
        D.map_tc_batch([mi], precision=precision)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ts = []
    for _ in range(reps):
        e0.record()
        D.map_tc_batch([mi], precision=precision)
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return float(np.median(ts))


def tune(precisions=('bf16x3', 'tf32', 'fp16'), mic_buckets=MIC_BUCKETS, item_buckets=('tiny', 'few', 'mid', 'many'),
         reps: int = 5, out: Path | str | None = TABLE_PATH, log=print) -> dict:
    """Time every candidate per shape class on cuda:0; write and return the table."""
    import torch
    dev = torch.device('cuda', 0)
    classes = {}
    t_start = time.perf_counter()
    for ib in item_buckets:
        side, nbins = REPRESENTATIVE[ib]
        for M in mic_buckets:
            mi = _instance(M, side, nbins, dev, seed=M)
            for prec in precisions:
                cands = candidates(M)
                times = {f'{pw}x{sp}': _time(mi, prec, (pw, sp), reps) for pw, sp in cands}
                best = min(times, key=times.get)
                dflt = next(f'{pw}x{sp}' for pw, sp in cands if sp == 1 and min(pw, -(-M // 16)) ==
                            min(DEFAULT[0], -(-M // 16)))
                pw, sp = (int(x) for x in best.split('x'))
                key = shape_class(M, side * side, nbins, prec)
                classes[key] = {'pass_chunks': pw, 'splits': sp, 'ms': times[best],
                                'default_ms': times[dflt],
                                'shape': {'mics': M, 'grid': side * side, 'bins': nbins}, 'candidates_ms': times}
                log(f'{key:24s} best {best:5s} {times[best]:8.3f} ms (default {times[dflt]:.3f} ms) | ' +
                    ' '.join(f'{c}={v:.3f}' for c, v in times.items()))
            del mi
            torch.cuda.empty_cache()
    table = {'device': torch.cuda.get_device_name(dev), 'reps': reps, 'seconds': time.perf_counter() - t_start,
             'classes': classes}
    if out is not None:
        Path(out).parent.mkdir(parents=True, exist_ok=True)
        Path(out).write_text(json.dumps(table, indent=1, sort_keys=True) + '\n')
        _load.cache_clear()
    return table


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description=__doc__.split('\n')[0])
    ap.add_argument('--out', default=str(TABLE_PATH))
    ap.add_argument('--reps', type=int, default=5)
    a = ap.parse_args(argv)
    tune(reps=a.reps, out=a.out)


if __name__ == '__main__':
    main()
