"""Block-wise spectra generators on the B200 (acoular/fprocess.py): ``RFFT``, ``AutoPowerSpectra``,
``CrossPowerSpectra``.

Same attributes, generator contract and block layout as the reference: ``result(num)`` yields
``(n, num_freqs * num_channels)`` numpy blocks of at most ``num`` snapshots, frequency-major with the
channels interlaced.  Each class also has ``result_device(num)``, which yields the same blocks as
``(n, num_freqs, channels...)`` device tensors; chained objects consume their source's device blocks,
so samples -> spectra -> auto/cross spectra never leave the GPU.  The FFT is the CSM path's FP64 kernel
(block sizes: powers of two, 16 ... 65536); the windows are those of ``BaseSpectra._get_source_data``.
``workers`` is accepted and ignored (there are no host FFT threads).
"""

from __future__ import annotations

import numpy as np
import torch
from scipy import fft

from . import _native as N
from . import device as D


def _device_blocks(source, num):
    """The source's blocks as device tensors (n, num_freqs, num_channels)."""
    if hasattr(source, 'result_device'):
        yield from source.result_device(num)
        return
    dev = D.require_cuda()
    nf, nc = source.num_freqs, source.num_channels
    for b in source.result(num):
        yield torch.as_tensor(np.ascontiguousarray(b)).to(dev).reshape(b.shape[0], nf, nc)


def _host_blocks(blocks):
    """Numpy blocks (n, rest...) of a generator of device blocks, as ``result(num)`` yields them.

    Each block is copied into page-locked host memory (torch's caching pinned allocator) on the copy stream
    and handed out one block later, so its download overlaps the computation of the next block.  Every
    yielded array is a block of its own; the pinned memory returns to the allocator's cache when the caller
    drops the array, so a consumer that handles one block at a time reuses the same few buffers instead of
    faulting in fresh host pages for every block.  Blocks above 1 GB are copied synchronously into ordinary
    host memory (the pinned allocator rounds sizes up to powers of two).
    """
    pending = None
    for b in blocks:
        if b.numel() * b.element_size() > (1 << 30):   # above 1 GB: a plain synchronous copy, no pinned block
            if pending is not None:
                pending[1].synchronize()
                yield pending[0].numpy().reshape(pending[0].shape[0], -1)
                pending = None
            yield b.cpu().numpy().reshape(b.shape[0], -1)
            continue
        dev = b.device
        compute = torch.cuda.current_stream(dev)
        copy = D.copy_stream(dev)
        ready = torch.cuda.Event()
        ready.record(compute)
        copy.wait_event(ready)
        host = torch.empty(b.shape, dtype=b.dtype, pin_memory=True)
        with torch.cuda.stream(copy):
            host.copy_(b, non_blocking=True)
            done = torch.cuda.Event()
            done.record(copy)
        b.record_stream(copy)
        if pending is not None:
            pending[1].synchronize()
            yield pending[0].numpy().reshape(pending[0].shape[0], -1)
        pending = (host, done)
    if pending is not None:
        pending[1].synchronize()
        yield pending[0].numpy().reshape(pending[0].shape[0], -1)


class RFFT:
    """One-sided FFT of real multichannel time data, block by block (acoular/fprocess.py:35-181)."""

    SCALINGS = ('none', 'energy', 'amplitude')

    def __init__(self, source=None, block_size: int = 1024, window: str = 'Rectangular', overlap: str = 'None',
                 precision: str = 'complex128', scaling: str = 'none', workers=None, device=None):
        self.source = source
        self.block_size = block_size
        if window not in D.WINDOWS:
            msg = f'window must be one of {tuple(D.WINDOWS)}, got {window!r}'
            raise ValueError(msg)
        if overlap not in D.OVERLAPS:
            msg = f'overlap must be one of {tuple(D.OVERLAPS)}, got {overlap!r}'
            raise ValueError(msg)
        if precision not in ('complex128', 'complex64'):
            msg = f"precision must be 'complex128' or 'complex64', got {precision!r}"
            raise ValueError(msg)
        if scaling not in self.SCALINGS:
            msg = f'scaling must be one of {self.SCALINGS}, got {scaling!r}'
            raise ValueError(msg)
        self.window = window
        self.overlap = overlap
        self.precision = precision
        self.scaling = scaling
        self.workers = workers
        self.device = device

    @property
    def block_size(self) -> int:
        return self._block_size

    @block_size.setter
    def block_size(self, value):
        if value % 2 != 0:
            msg = 'Block size must be even'
            raise ValueError(msg)
        self._block_size = int(value)

    @property
    def num_freqs(self) -> int:
        return int(self.block_size / 2 + 1)

    @property
    def num_channels(self) -> int:
        return self.source.num_channels

    @property
    def sample_freq(self) -> float:
        return self.source.sample_freq

    @property
    def num_samples(self) -> int:
        if self.source.num_samples >= 0:
            return int(np.floor(self.source.num_samples / self.block_size))
        return -1

    @property
    def freqs(self) -> np.ndarray:
        if self.source is not None:
            return abs(fft.fftfreq(self.block_size, 1.0 / self.source.sample_freq)[: int(self.block_size / 2 + 1)])
        return np.array([])

    @property
    def digest(self) -> str:
        src = getattr(self.source, 'digest', id(self.source))
        return f'rfft|{src}|{self.scaling}|{self.precision}|{self.block_size}|{self.window}|{self.overlap}'

    def _scale_value(self) -> float:
        wind = D.WINDOWS[self.window](self.block_size)
        if self.scaling in ('none', 'energy'):
            return 1 / np.sqrt(np.dot(wind, wind) / self.block_size)
        return 1 / wind.sum()

    def _samples(self):
        ps = _SampleSource(self.source)
        return ps.samples_device(self.device)

    def result_device(self, num: int = 1):
        """Blocks of at most ``num`` spectra as device tensors (n, num_freqs, num_channels)."""
        N_ = self.block_size
        if N_ < 16 or N_ > 65536 or N_ & (N_ - 1):
            msg = f'block_size {N_}: the FFT kernel takes powers of two from 16 to 65536'
            raise ValueError(msg)
        x = self._samples()
        dev = x.device
        S, M = x.shape
        ov = D.OVERLAPS[self.overlap]
        hop = N_ // ov
        K = D.num_windows(S, N_, ov)
        F = self.num_freqs
        win, _ = D.window_vector(self.window, N_, dev)
        tw = D.twiddles(N_, dev)
        prec = N.C64 if self.precision == 'complex64' else N.C128
        cdt = torch.complex64 if self.precision == 'complex64' else torch.complex128
        scale = float(self._scale_value())
        twice = int(self.scaling in ('amplitude', 'energy'))
        sdt = N.F32 if x.dtype == torch.float32 else N.F64
        if K == 0:
            if num > 1:   # the reference yields one row of zeros when there is no complete block
                yield torch.zeros((1, F, M), dtype=cdt, device=dev)
            return
        num = int(num)
        ws = None
        for w0 in range(0, K, num):
            n = min(num, K - w0)
            out = torch.empty((n, F, M), dtype=cdt, device=dev)
            for s0 in range(0, n, 65535):        # one launch covers at most 65535 windows
                m = min(65535, n - s0)
                need = N.lib().acb_spectra_workspace_bytes(M, N_, m)
                if ws is None or ws.numel() < need:
                    ws = torch.empty(need, dtype=torch.uint8, device=dev)
                N.check(N.lib().acb_spectra(x.data_ptr(), sdt, S, M, N_, hop, w0 + s0, m, win.data_ptr(),
                                            tw.data_ptr(), prec, scale, twice, out[s0:s0 + m].data_ptr(),
                                            ws.data_ptr(), ws.numel(), N.stream_handle()), 'acb_spectra')
            yield out

    def result(self, num: int = 1):
        yield from _host_blocks(self.result_device(num))


class AutoPowerSpectra:
    """Real auto-power spectra |X|^2 of a spectra source (acoular/fprocess.py:286-366)."""

    def __init__(self, source=None, scaling: str = 'power', single_sided: bool = True, precision: str = 'float64'):
        if scaling not in ('power', 'psd'):
            msg = f"scaling must be 'power' or 'psd', got {scaling!r}"
            raise ValueError(msg)
        self._check_precision(precision)
        self.source = source
        self.scaling = scaling
        self.single_sided = bool(single_sided)
        self.precision = precision

    @staticmethod
    def _check_precision(precision):
        if precision not in ('float64', 'float32'):
            msg = f"precision must be 'float64' or 'float32', got {precision!r}"
            raise ValueError(msg)

    @property
    def block_size(self) -> int:
        return self.source.block_size

    @property
    def num_freqs(self) -> int:
        return self.source.num_freqs

    @property
    def num_channels(self) -> int:
        return self.source.num_channels

    @property
    def sample_freq(self) -> float:
        return self.source.sample_freq

    @property
    def digest(self) -> str:
        src = getattr(self.source, 'digest', id(self.source))
        return f'{type(self).__name__}|{src}|{self.precision}|{self.scaling}|{self.single_sided}'

    def _get_scaling_value(self) -> float:
        scale = 1 / self.block_size**2
        if self.single_sided:
            scale *= 2
        if self.scaling == 'psd':
            scale *= self.block_size * self.source.sample_freq
        return scale

    def result_device(self, num: int = 1):
        scale = float(self._get_scaling_value())
        odt = torch.float32 if self.precision == 'float32' else torch.float64
        for b in _device_blocks(self.source, num):
            b = b.contiguous()
            prec = N.C64 if b.dtype == torch.complex64 else N.C128
            out = torch.empty(b.shape, dtype=odt, device=b.device)
            N.check(N.lib().acb_auto_spectra(b.data_ptr(), b.numel(), prec, int(odt == torch.float32), scale,
                                             out.data_ptr(), N.stream_handle()), 'acb_auto_spectra')
            yield out

    def result(self, num: int = 1):
        yield from _host_blocks(self.result_device(num))


class CrossPowerSpectra(AutoPowerSpectra):
    """Per-snapshot cross-spectral matrices of a spectra source, flattened (acoular/fprocess.py:369-467).

    ``calc_mode='full'`` gives the whole matrix of every bin.  ``'upper'`` and ``'lower'`` behave as the
    reference's do: they return the one element for a single channel, and for more channels the
    reference's own block assignment fails with a ``ValueError``, which is raised here too.
    """

    def __init__(self, source=None, scaling: str = 'power', single_sided: bool = True,
                 precision: str = 'complex128', calc_mode: str = 'full'):
        if calc_mode not in ('full', 'upper', 'lower'):
            msg = f"calc_mode must be 'full', 'upper' or 'lower', got {calc_mode!r}"
            raise ValueError(msg)
        super().__init__(source=source, scaling=scaling, single_sided=single_sided, precision='float64')
        if precision not in ('complex128', 'complex64'):
            msg = f"precision must be 'complex128' or 'complex64', got {precision!r}"
            raise ValueError(msg)
        self.precision = precision
        self.calc_mode = calc_mode

    @property
    def num_channels(self) -> int:
        n = self.source.num_channels
        return n**2 if self.calc_mode == 'full' else int(n + n * (n - 1) / 2)

    @property
    def digest(self) -> str:
        return super().digest + f'|{self.calc_mode}'

    def result_device(self, num: int = 1):
        """Blocks (n, num_freqs, M, M) of per-snapshot matrices on the device (``calc_mode='full'``)."""
        scale = float(self._get_scaling_value())
        cdt = torch.complex64 if self.precision == 'complex64' else torch.complex128
        prec = N.C64 if cdt == torch.complex64 else N.C128
        M = self.source.num_channels
        if self.calc_mode != 'full' and M > 1:
            msg = (f"calc_mode '{self.calc_mode}' with {M} channels: the reference cannot assign its "
                   f'(num_freqs, {M}, {M}) triangle block to a row of {self.num_channels * self.num_freqs} values')
            raise ValueError(msg)
        for b in _device_blocks(self.source, num):
            x = b.to(cdt).contiguous()
            n, F = x.shape[0], x.shape[1]
            out = torch.empty((n, F, M, M), dtype=cdt, device=x.device)
            N.check(N.lib().acb_cross_spectra(x.data_ptr(), n, F, M, prec, scale, out.data_ptr(), N.stream_handle()),
                    'acb_cross_spectra')
            yield out

    def result(self, num: int = 1):
        yield from _host_blocks(self.result_device(num))


class _SampleSource:
    """The source's samples as a device tensor, as PowerSpectra takes them."""

    def __init__(self, source):
        self.source = source

    def samples_device(self, device=None) -> torch.Tensor:
        from .spectra import PowerSpectra
        ps = PowerSpectra(source=self.source, device=device)
        return ps._samples_device()
