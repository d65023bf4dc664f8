"""Seeded synthetic workloads with the shapes of the published benchmark configurations.

No public dataset is involved: every workload is seeded synthetic data.

* :func:`three_sources_64`  -- 64 mics in a 0.5 m disk, three white-noise monopoles at z=-0.3 m,
  51,200 samples at 51.2 kHz, block 128 / Hanning / 50 %, 41x41 grid, 8 kHz third-octave band.
* :func:`precision_256`     -- 256 mics in a 1 m disk, 8 monopoles (seeds 1-8, rms log-uniform over
  20 dB) at z=-1 m, 10 s float32 at 51.2 kHz, block 1024 / Hanning / 50 %, all 513 bins,
  401x401 grid over [-1, 1]^2 at z=-1 m.
* :func:`large_3d`          -- 1024-mic log spiral (2 m), block 4096, 16 s float32, 200 bins in
  1-16 kHz, 101x101x41 RectGrid3D over [-1,1]^2 x [0.5,1.5] m, 20 monopoles.
* :func:`batched_instances` -- 64 uneven instances (mics 32..256, grids 21^2..301^2, blocks
  256..2048, 1..40 sources, 30 bins each).
* :func:`serving_requests`  -- request stream for the serving loop (64..512 mics, 41^2..201^2 grids,
  0.1 s of samples, one third-octave band).

Small workloads use the host :class:`~acoular_b200.sources.PointSource` restatement; large ones use
:func:`monopole_time_data_torch`, the same monopole model (x16 resampled signal, nearest emission
index, 1/r) evaluated on the GPU so that multi-GB inputs are generated in seconds.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .grids import RectGrid, RectGrid3D
from .microphones import MicGeom, disk_mics, log_spiral_mics
from .sources import Mixer, PointSource, WNoiseGenerator

FS = 51200.0
STEER_TYPES = ('classic', 'inverse', 'true level', 'true location')


@dataclass
class Workload:
    name: str
    mics: MicGeom
    grid: object
    locs: list
    seeds: list
    rms: list
    fs: float
    num_samples: int
    block_size: int
    window: str = 'Hanning'
    overlap: str = '50%'
    precision: str = 'complex128'
    c: float = 343.0
    band: tuple | None = None          # (center frequency, 1/n octave)
    bins: np.ndarray | None = None     # explicit bin subset
    steer_type: str = 'true level'
    r_diag: bool = True
    dtype: str = 'float64'
    correlated_pairs: list = field(default_factory=list)

    def time_data(self) -> np.ndarray:
        """Host generation through the PointSource/Mixer restatement (small workloads)."""
        srcs = []
        for loc, seed, rms in zip(self.locs, self.seeds, self.rms):
            sig = WNoiseGenerator(sample_freq=self.fs, num_samples=self.num_samples, seed=seed, rms=rms)
            srcs.append(PointSource(signal=sig, mics=self.mics, loc=loc))
        mix = Mixer(srcs[0], srcs[1:])
        data = np.concatenate([b.copy() for b in mix.result(4096)])
        return data.astype(self.dtype, copy=False)


def three_sources_64() -> Workload:
    return Workload(
        name='three_sources_64mic_41x41',
        mics=disk_mics(64, 0.5, seed=1),
        grid=RectGrid(x_min=-0.2, x_max=0.2, y_min=-0.2, y_max=0.2, z=-0.3, increment=0.01),
        locs=[(-0.1, -0.1, -0.3), (0.15, 0.0, -0.3), (0.0, 0.1, -0.3)],
        seeds=[1, 2, 3], rms=[1.0, 0.7, 0.5], fs=FS, num_samples=51200, block_size=128,
        band=(8000.0, 3))


def precision_256() -> Workload:
    rng = np.random.RandomState(2024)
    locs = [(rng.uniform(-0.8, 0.8), rng.uniform(-0.8, 0.8), -1.0) for _ in range(8)]
    rms = list(10 ** (-rng.uniform(0, 20, size=8) / 20))
    return Workload(
        name='precision_256mic_401x401_513bins',
        mics=disk_mics(256, 1.0, seed=2),
        grid=RectGrid(x_min=-1.0, x_max=1.0, y_min=-1.0, y_max=1.0, z=-1.0, increment=0.005),
        locs=locs, seeds=list(range(1, 9)), rms=rms, fs=FS, num_samples=512000, block_size=1024,
        dtype='float32')


def large_3d() -> Workload:
    rng = np.random.RandomState(4096)
    locs = [(rng.uniform(-0.9, 0.9), rng.uniform(-0.9, 0.9), rng.uniform(0.55, 1.45)) for _ in range(20)]
    seeds = list(range(101, 121))
    # ten correlated pairs: sources 2j and 2j+1 share one signal generator
    for j in range(5):
        seeds[2 * j + 1] = seeds[2 * j]
    rms = list(10 ** (-rng.uniform(0, 12, size=20) / 20))
    freqs = np.abs(np.fft.fftfreq(4096, 1 / FS)[:2049])
    lo, hi = np.searchsorted(freqs, 1000.0), np.searchsorted(freqs, 16000.0)
    bins = np.unique(np.linspace(lo, hi, 200).round().astype(int))
    return Workload(
        name='large3d_1024mic_101x101x41_200bins',
        mics=log_spiral_mics(1024, 2.0, seed=4),
        grid=RectGrid3D(x_min=-1.0, x_max=1.0, y_min=-1.0, y_max=1.0, z_min=0.5, z_max=1.5,
                        increment=(0.02, 0.02, 0.025)),
        locs=locs, seeds=seeds, rms=rms, fs=FS, num_samples=819200, block_size=4096, bins=bins,
        steer_type='true location', r_diag=True, dtype='float32')


def batched_instances(n: int = 64, seed: int = 3):
    """Uneven instances: mics {32,64,128,256}, square grids 21^2..301^2, blocks 256..2048, 30 bins."""
    rng = np.random.RandomState(seed)
    out = []
    for i in range(n):
        M = int(rng.choice([32, 64, 128, 256]))
        side = int(rng.randint(21, 302))
        z = float(rng.uniform(0.5, 2.0))
        N = int(rng.choice([256, 512, 1024, 2048]))
        nsrc = int(rng.randint(1, 41))
        locs = [(rng.uniform(-0.5, 0.5), rng.uniform(-0.5, 0.5), z) for _ in range(nsrc)]
        F = N // 2 + 1
        b0 = int(rng.randint(1, F - 30))
        inc = 1.0 / (side - 1)
        out.append(Workload(
            name=f'inst{i}', mics=disk_mics(M, 0.5, seed=100 + i),
            grid=RectGrid(x_min=-0.5, x_max=0.5, y_min=-0.5, y_max=0.5, z=z, increment=inc),
            locs=locs, seeds=list(range(1000 * i, 1000 * i + nsrc)), rms=list(rng.uniform(0.3, 1.0, nsrc)),
            fs=FS, num_samples=N * 16, block_size=N, precision='complex64', bins=np.arange(b0, b0 + 30),
            dtype='float32'))
    return out


def monopole_time_data_torch(wl: Workload, device='cuda', chunk: int = 65536):
    """Monopole mixture on the GPU: x16 Fourier-resampled white noise, nearest emission index, 1/r.

    Same model as :class:`~acoular_b200.sources.PointSource`; float64 index arithmetic, output in
    ``wl.dtype``.  Returns a device tensor ``(num_samples, num_mics)``.
    """
    import torch
    from scipy.signal import resample

    up = 16
    mpos = torch.as_tensor(wl.mics.pos, dtype=torch.float64, device=device)
    out = torch.zeros((wl.num_samples, wl.mics.num_mics), dtype=torch.float64, device=device)
    cache = {}
    for loc, seed, rms in zip(wl.locs, wl.seeds, wl.rms):
        if seed not in cache:
            sig = WNoiseGenerator(sample_freq=wl.fs, num_samples=wl.num_samples, seed=seed, rms=1.0)
            cache[seed] = torch.as_tensor(resample(sig.signal(), up * wl.num_samples), device=device)
        usig = cache[seed] * rms
        n_sig = usig.shape[0]
        d = mpos - torch.as_tensor(np.asarray(loc, float).reshape(3, 1), device=device)
        rm = torch.sqrt((d * d).sum(0))
        ind0 = (-rm / wl.c) * wl.fs * up
        for t0 in range(0, wl.num_samples, chunk):
            t = torch.arange(t0, min(t0 + chunk, wl.num_samples), device=device, dtype=torch.float64)
            idx = torch.floor(0.5 + ind0[None, :] + up * t[:, None]).to(torch.int64)
            idx = torch.remainder(idx, n_sig)
            out[t0:t0 + t.shape[0]] += usig[idx] / rm[None, :]
    return out.to(torch.float32 if wl.dtype == 'float32' else torch.float64)
