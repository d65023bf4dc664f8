"""``PowerSpectra`` with the CSM computed on the B200 (acoular/spectra.py:52-588).

Same attributes and semantics as the reference: ``block_size`` (128 ... 65536; blocks above 16384
samples take the FFT as interleaved 8192-point sub-transforms and a combining pass), ``window``, ``overlap``, ``precision`` ('complex128' | 'complex64'),
``fftfreq()``, ``num_blocks`` (the reference's float formula), ``csm`` (lazy, recomputed when
the source or a setting changes), ``indices`` / ``ind_low`` / ``ind_high`` / ``freq_range``,
``eigvals`` / ``eigvecs``.  ``calc_csm()`` returns the complex128 (F, M, M) numpy array the
reference returns; ``csm_device`` keeps the same matrix resident on the GPU for the beamformer.
HDF5 result caching (``cached`` / ``config.global_caching``) is not implemented: every setting
behaves like ``global_caching='none'``.

Two settings have no counterpart in the reference: ``form`` ('f64', the default, the reference's
arithmetic; or 'tc', the Welch Gram on the tensor cores) and ``tc_precision`` ('tf32' or 'bf16x3',
the operand form of the tensor-core Gram).  Either way the CSM is complex128.
"""

from __future__ import annotations

import numpy as np
import torch
from scipy import fft

from . import device as D

BLOCK_SIZES = (1024, 128, 256, 512, 2048, 4096, 8192, 16384, 32768, 65536)


class PowerSpectra:
    def __init__(self, source=None, block_size: int = 1024, window: str = 'Rectangular', overlap: str = 'None',
                 precision: str = 'complex128', cached: bool = False, ind_low: int | None = None,
                 ind_high: int | None = None, device=None, form: str = 'f64', tc_precision: str = 'tf32'):
        self.source = source
        self.form = form
        self.tc_precision = tc_precision
        self.block_size = block_size
        self.window = window
        self.overlap = overlap
        self.precision = precision
        self.cached = cached
        self._ind_low = 1 if ind_low is None else ind_low
        self._ind_high = -1 if ind_high is None else ind_high
        self._freqlc, self._freqhc = 0.0, 0.0
        self._index_set_last = True
        self.device = device
        self._cache_key = None
        self._csm_dev = None
        self._csm_host = None
        self._evd = None

    # --- validated settings (traits Enum / Map semantics) -------------------------------------
    def __setattr__(self, name, value):
        if name == 'block_size' and value not in BLOCK_SIZES:
            msg = f'block_size must be one of {BLOCK_SIZES}, got {value!r}'
            raise ValueError(msg)
        if name == 'window' and value not in D.WINDOWS:
            msg = f'window must be one of {tuple(D.WINDOWS)}, got {value!r}'
            raise ValueError(msg)
        if name == 'overlap' and value not in D.OVERLAPS:
            msg = f'overlap must be one of {tuple(D.OVERLAPS)}, got {value!r}'
            raise ValueError(msg)
        if name == 'precision' and value not in ('complex128', 'complex64'):
            msg = f"precision must be 'complex128' or 'complex64', got {value!r}"
            raise ValueError(msg)
        if name == 'form' and value not in ('f64', 'tc'):
            msg = f"form must be 'f64' or 'tc', got {value!r}"
            raise ValueError(msg)
        if name == 'tc_precision' and value not in ('tf32', 'bf16x3'):
            msg = f"tc_precision must be 'tf32' or 'bf16x3', got {value!r}"
            raise ValueError(msg)
        object.__setattr__(self, name, value)

    @property
    def overlap_(self) -> int:
        return D.OVERLAPS[self.overlap]

    @property
    def window_(self):
        return D.WINDOWS[self.window]

    @property
    def sample_freq(self):
        return self.source.sample_freq

    @property
    def num_channels(self):
        return self.source.num_channels

    @property
    def num_blocks(self) -> float:
        return D.num_blocks(self.source.num_samples, self.block_size, self.overlap_)

    @property
    def digest(self) -> str:
        src = getattr(self.source, 'digest', id(self.source))
        tc = f'|tc-{self.tc_precision}' if self.form == 'tc' else ''
        return f'{src}|{self.block_size}|{self.window}|{self.overlap}|{self.precision}{tc}'

    def fftfreq(self):
        if self.source is not None:
            return abs(fft.fftfreq(self.block_size, 1.0 / self.source.sample_freq)[: int(self.block_size / 2 + 1)])
        return None

    # --- frequency range (acoular/spectra.py:285-341) ------------------------------------------
    @property
    def ind_low(self):
        f = self.fftfreq()
        if f is None:
            return 0
        if self._index_set_last:
            return min(self._ind_low, f.shape[0] - 1)
        return int(np.searchsorted(f[:-1], self._freqlc))

    @ind_low.setter
    def ind_low(self, v):
        self._index_set_last = True
        self._ind_low = v

    @property
    def ind_high(self):
        f = self.fftfreq()
        if f is None:
            return None
        if self._index_set_last:
            if self._ind_high is None:
                return None
            return min(self._ind_high, f.shape[0] - 1)
        if self._freqhc is None:
            return None
        return int(np.searchsorted(f[:-1], self._freqhc))

    @ind_high.setter
    def ind_high(self, v):
        self._index_set_last = True
        self._ind_high = v

    @property
    def freq_range(self):
        f = self.fftfreq()
        if f is None:
            return None
        if self.ind_high is None:
            return np.array([f[self.ind_low], None])
        return f[[self.ind_low, self.ind_high]]

    @freq_range.setter
    def freq_range(self, fr):
        if fr is not None:
            self._index_set_last = False
            self._freqlc, self._freqhc = fr[0], fr[1]

    @property
    def indices(self):
        f = self.fftfreq()
        if f is None:
            return None
        idx = np.arange(f.shape[0], dtype=int)
        if self.ind_high is None:
            return idx[self.ind_low:]
        return idx[self.ind_low:self.ind_high]

    # --- CSM ------------------------------------------------------------------------------------
    def _device(self):
        return D.require_cuda(self.device)

    def _samples_host_or_device(self) -> torch.Tensor:
        """The source samples as a (S, M) float32/float64 tensor, wherever they live."""
        t = self.source
        data = getattr(t, 'data', None)
        if data is None:
            data = t.as_array()
        if isinstance(data, torch.Tensor):
            x = data
        else:
            arr = np.ascontiguousarray(data)
            if arr.dtype not in (np.float32, np.float64):
                arr = arr.astype(np.float64)
            x = torch.from_numpy(arr)
        if x.dtype not in (torch.float32, torch.float64):
            x = x.to(torch.float64)
        return x

    def _samples_device(self) -> torch.Tensor:
        x = self._samples_host_or_device()
        if x.device.type == 'cpu':
            x = x.to(self._device(), non_blocking=x.is_pinned())
        return x.contiguous()

    def _csm_streamed(self, x: torch.Tensor, prec: str, nchunks: int = 8) -> torch.Tensor:
        """CSM of pinned host samples: the samples go to the device in chunks of windows on a copy
        stream, and each chunk's Welch sums are accumulated as soon as its rows have landed, so the
        upload overlaps the FFT and Gram of the previous chunks.  Same sums as one pass."""
        dev = self._device()
        S, M = x.shape
        N = self.block_size
        ov = D.OVERLAPS[self.overlap]
        hop = N // ov
        K = D.num_windows(S, N, ov)
        F = N // 2 + 1
        xd = torch.empty((S, M), dtype=x.dtype, device=dev)
        cdt = torch.complex64 if prec == 'complex64' else torch.complex128
        up = torch.zeros((F, M, M), dtype=cdt, device=dev)
        compute = torch.cuda.current_stream(dev)
        copy = D.copy_stream(dev)
        copy.wait_stream(compute)              # xd is ready for writing
        per = -(-K // nchunks)                 # windows per chunk, in whole blocks of 32
        wc = max(32, (per + 31) // 32 * 32)
        rows = 0
        for w0 in range(0, max(K, 1), wc):
            w1 = min(K, w0 + wc)
            need = S if w1 >= K else (w1 - 1) * hop + N
            if need > rows:
                with torch.cuda.stream(copy):
                    xd[rows:need].copy_(x[rows:need], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(copy)
                compute.wait_event(ev)
                rows = need
            if w1 > w0:
                D.csm_upper_accumulate(xd, N, self.window, self.overlap, prec, csm_upper=up, first_window=w0,
                                       windows=w1 - w0)
        _, weight = D.window_vector(self.window, N, dev)
        with np.errstate(divide='ignore', invalid='ignore'):
            scale = np.float64(2.0 / N) / np.float64(weight) / np.float64(D.num_blocks(S, N, ov))
        return D.csm_finalize(up, float(scale))

    def calc_csm_device(self) -> torch.Tensor:
        """The CSM (F, M, M) complex128 as a device tensor (see :meth:`calc_csm`)."""
        t = self.source
        if t.num_samples == -1:
            msg = 'PowerSpectra requires a finite source'
            raise ValueError(msg)
        prec = f'tc_{self.tc_precision}' if self.form == 'tc' else self.precision
        x = self._samples_host_or_device()
        if x.device.type == 'cpu' and x.is_pinned() and x.is_contiguous() and x.numel() >= (1 << 22):
            return self._csm_streamed(x, prec)
        x = self._samples_device()
        return D.calc_csm(x, self.block_size, self.window, self.overlap, prec)

    def calc_csm(self) -> np.ndarray:
        """CSM of the source for all ``block_size/2 + 1`` bins, (F, M, M) complex128."""
        return self.calc_csm_device().cpu().numpy()

    def _refresh(self):
        key = self.digest
        if key != self._cache_key:
            self._cache_key = key
            self._csm_dev = None
            self._csm_host = None
            self._evd = None

    @property
    def csm_device(self) -> torch.Tensor:
        self._refresh()
        if self._csm_dev is None:
            self._csm_dev = self.calc_csm_device()
        return self._csm_dev

    @property
    def csm(self) -> np.ndarray:
        self._refresh()
        if self._csm_host is None:
            self._csm_host = self.csm_device.cpu().numpy()
        return self._csm_host

    # --- eigen-decomposition (acoular/spectra.py:351-364) ---------------------------------------
    @property
    def evd_device(self):
        """``(eigvals (F, M) float64, eigvecs (F, M, M) complex128)`` of the CSM on the device: the
        library's batched Hermitian eigendecomposition (``acb_heevd_f64``), eigenvalues ascending as numpy
        returns them.  The eigenvector phases may differ from LAPACK's; the eigenvalue beamformers depend on
        them only through |v^H h|."""
        self._refresh()
        if getattr(self, '_evd_dev', None) is None or self._evd_dev[0] != self._cache_key:
            ev, evec, info = D.heevd_f64(self.csm_device)
            if int(info.max()):
                msg = 'acb_heevd_f64: the QL iteration did not converge for some bins'
                raise RuntimeError(msg)
            self._evd_dev = (self._cache_key, ev, evec)
        return self._evd_dev[1], self._evd_dev[2]

    # host LAPACK, as the reference
    def _get_evd(self):
        self._refresh()
        if self._evd is None:
            dt = 'float64' if self.precision == 'complex128' else 'float32'
            csm = self.csm
            ev = np.empty(csm.shape[0:2], dtype=dt)
            evec = np.empty(csm.shape, dtype=self.precision)
            for i in range(csm.shape[0]):
                ev[i], evec[i] = np.linalg.eigh(csm[i])
            self._evd = (ev, evec)
        return self._evd

    @property
    def eigvals(self):
        return self._get_evd()[0]

    @property
    def eigvecs(self):
        return self._get_evd()[1]


class PowerSpectraImport(PowerSpectra):
    """A given CSM (F, M, M) with its frequencies (acoular/spectra.py:591-697)."""

    def __init__(self, csm=None, frequencies=None, device=None):
        object.__setattr__(self, 'block_size', 1024)
        super().__init__(source=None, device=device)
        # all lines of an imported CSM count: first index 0, no last index (acoular/spectra.py:667-668)
        self._ind_low, self._ind_high = 0, None
        self._import_csm = None
        self._frequencies = None
        self.set_csm(csm, frequencies)

    def set_csm(self, csm, frequencies):
        if csm is None:
            return
        csm = np.asarray(csm)
        if csm.ndim != 3 or csm.shape[1] != csm.shape[2]:
            msg = 'The cross spectral matrix must have the following shape: (number of frequencies, num_channels, num_channels)!'
            raise ValueError(msg)
        self._import_csm = csm
        self._frequencies = np.atleast_1d(np.asarray(frequencies, dtype=float))
        self._cache_key = None

    @property
    def num_channels(self):
        return self._import_csm.shape[1]

    @property
    def digest(self) -> str:
        c = self._import_csm
        return f'import|{id(c)}|{c.shape if c is not None else None}'

    def fftfreq(self):
        return self._frequencies

    def calc_csm_device(self) -> torch.Tensor:
        return torch.as_tensor(np.ascontiguousarray(self._import_csm, dtype=np.complex128), device=self._device())

    def calc_csm(self) -> np.ndarray:
        return self._import_csm
