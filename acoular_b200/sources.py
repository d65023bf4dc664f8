"""Time-signal sources: recorded data and the simulation generators used to make seeded inputs.

* :class:`TimeSamples`     -- array-backed source, ``result(num)`` as acoular/sources.py:417-467
* :class:`WNoiseGenerator` -- white noise, acoular/signals.py:255-269 (``RandomState(seed)``)
* :class:`PointSource`     -- stationary monopole, acoular/sources.py:637-841 (``prepadding='loop'``)
* :class:`Mixer`           -- sum of sources, acoular/tprocess.py:1561-1607

The simulation classes reproduce the reference's arithmetic (x16 Fourier resampling, nearest-index
lookup with sequentially accumulated emission indices, division by the distance) so that the seeded
inputs of the benchmark workloads have the reference's value distribution.  They are host-side
helpers; the beamforming path itself starts at the sample array.
"""

from __future__ import annotations

import hashlib

import numpy as np
from scipy.signal import resample

from .environments import Environment
from .microphones import MicGeom


class SamplesGenerator:
    """Common interface: ``sample_freq``, ``num_channels``, ``num_samples`` and ``result(num)``."""

    sample_freq: float
    num_channels: int
    num_samples: int

    def result(self, num):  # pragma: no cover - interface
        raise NotImplementedError

    def as_array(self) -> np.ndarray:
        """All samples as one ``(num_samples, num_channels)`` array."""
        return np.concatenate([np.array(b, copy=True) for b in self.result(max(1, min(self.num_samples, 65536)))])


class TimeSamples(SamplesGenerator):
    """Multichannel time data held in memory, shape ``(num_samples, num_channels)``."""

    def __init__(self, data=None, sample_freq: float = 1.0):
        if data is None or hasattr(data, 'data_ptr'):
            self.data = data  # None or a torch tensor (kept as is, e.g. pinned host memory)
        else:
            self.data = np.asarray(data)
        self.sample_freq = float(sample_freq)

    @property
    def num_samples(self) -> int:
        return 0 if self.data is None else self.data.shape[0]

    @property
    def num_channels(self) -> int:
        return 0 if self.data is None else self.data.shape[1]

    @property
    def digest(self) -> str:
        """Identifier of the data: content hash of evenly spaced whole sample rows (about 128 KB, the last
        row included) with the shape, dtype and sample rate, computed once per array object.  Only the
        sampled rows leave the device when the data is a CUDA tensor.

        Replace ``data`` (assign a new array) after changing samples in place."""
        key = (id(self.data), None if self.data is None else (tuple(self.data.shape), str(self.data.dtype)),
               self.sample_freq)
        if getattr(self, '_digest_key', None) != key:
            h = hashlib.blake2b(digest_size=16)
            if self.data is not None:
                a = self.data
                if not hasattr(a, 'detach'):
                    a = np.asarray(a)
                shape = tuple(a.shape)
                h.update(str((shape, str(a.dtype), self.sample_freq)).encode())
                if a.ndim >= 1 and shape[0] > 0:
                    row_bytes = max(1, a[0].numel() * a.element_size() if hasattr(a, 'detach') else a[0].nbytes)
                    step = max(1, shape[0] * row_bytes // (128 << 10))
                    rows = a[::step]
                    last = a[shape[0] - 1:]
                    if hasattr(a, 'detach'):
                        rows, last = rows.detach().cpu().numpy(), last.detach().cpu().numpy()
                    h.update(np.ascontiguousarray(rows).tobytes())
                    h.update(np.ascontiguousarray(last).tobytes())
                else:
                    h.update(np.ascontiguousarray(a.detach().cpu().numpy() if hasattr(a, 'detach') else a).tobytes())
            self._digest = '_' + h.hexdigest()
            self._digest_key = key
        return self._digest

    def result(self, num=128):
        if self.num_samples == 0:
            msg = 'no samples available'
            raise OSError(msg)
        i = 0
        while i < self.num_samples:
            yield self.data[i:num + i]
            i += num

    def as_array(self) -> np.ndarray:
        return self.data


class WNoiseGenerator:
    """Gaussian white noise ``rms * RandomState(seed).standard_normal(num_samples)``."""

    def __init__(self, sample_freq: float = 1.0, num_samples: int = 0, seed: int = 0, rms: float = 1.0):
        self.sample_freq = float(sample_freq)
        self.num_samples = int(num_samples)
        self.seed = int(seed)
        self.rms = float(rms)

    def signal(self) -> np.ndarray:
        return self.rms * np.random.RandomState(self.seed).standard_normal(self.num_samples)

    def usignal(self, factor: int) -> np.ndarray:
        """Fourier resampling to ``factor`` times the sample rate (acoular/signals.py:93-126)."""
        return resample(self.signal(), factor * self.num_samples)


class PointSource(SamplesGenerator):
    """Stationary monopole emitting ``signal``; output ``(num, num_mics)`` blocks."""

    def __init__(self, signal: WNoiseGenerator, mics: MicGeom, loc=(0.0, 0.0, 1.0), env: Environment | None = None,
                 start_t: float = 0.0, start: float = 0.0, up: int = 16):
        self.signal = signal
        self.mics = mics
        self.loc = np.asarray(loc, dtype=float).reshape((3, 1))
        self.env = env if env is not None else Environment()
        self.start_t = float(start_t)
        self.start = float(start)
        self.up = int(up)

    @property
    def num_samples(self) -> int:
        return self.signal.num_samples

    @property
    def sample_freq(self) -> float:
        return self.signal.sample_freq

    @property
    def num_channels(self) -> int:
        return self.mics.num_mics

    def result(self, num=128):
        num_est = self.num_samples + (self.start_t - self.start) * self.sample_freq
        nblocks = int(np.ceil(num_est / num))
        signal = self.signal.usignal(self.up)
        rm = self.env.apparent_r(self.loc, self.mics.pos).reshape(1, -1)
        ind = (-rm / self.env.c - self.start_t + self.start) * self.sample_freq * self.up
        n_sig = signal.shape[0]
        out = np.empty((num, self.num_channels))
        for blk in range(nblocks):
            bs = num if blk < nblocks - 1 else (self.num_samples % num or num)
            # ind advances by `up` once per output row, accumulated sequentially like the reference
            steps = np.empty((bs + 1, ind.shape[1]))
            steps[0] = ind[0]
            steps[1:] = self.up
            acc = np.add.accumulate(steps, axis=0)
            idx = (0.5 + acc[:bs]).astype(np.int64)
            idx = np.where(idx < 0, idx + n_sig, idx)  # negative indices wrap ('loop' prepadding)
            out[:bs] = signal[idx] / rm[0]
            ind = acc[bs:bs + 1].copy()
            yield out[:bs]


class Mixer(SamplesGenerator):
    """Sum of a primary source and further sources, block by block."""

    def __init__(self, source: SamplesGenerator, sources=()):
        self.source = source
        self.sources = list(sources)

    @property
    def num_samples(self) -> int:
        return self.source.num_samples

    @property
    def sample_freq(self) -> float:
        return self.source.sample_freq

    @property
    def num_channels(self) -> int:
        return self.source.num_channels

    def result(self, num):
        gens = [s.result(num) for s in self.sources]
        for temp in self.source.result(num):
            sh = temp.shape[0]
            for g in gens:
                try:
                    temp1 = next(g)
                except StopIteration:
                    return
                if temp.shape[0] > temp1.shape[0]:
                    temp = temp[: temp1.shape[0]]
                temp += temp1[: temp.shape[0]]
            yield temp
            if sh > temp.shape[0]:
                break
