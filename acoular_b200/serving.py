"""Continuous-batching beamforming server on one GPU.

Requests carry a block of multichannel samples for a *stream*; a stream is one array with a fixed
geometry, grid, FFT block size and frequency band.  The server keeps, per stream and on the device:

* the running Welch sum of the CSM (upper triangle) over everything the stream has sent, for the
  band's bins only, plus the samples of the not yet complete window (so windows span request
  boundaries exactly as ``PowerSpectra`` windows a continuous recording, acoular/spectra.py:171-184);
* its geometry and grid (shared by streams that use the same ones);
* its finished CSM, map and band-map buffers, and pinned host buffers for the samples coming in and
  the band map going out -- so serving a request allocates no pinned host memory (a pinned
  allocation on the request path stalled the worker for 100-250 ms at a time).

A worker thread takes every request that is pending when the GPU becomes free (continuous
batching: requests that arrive during a batch join the next one), updates each stream's CSM with
the new samples, finishes the CSMs, and computes all the maps in one batched tensor-core launch
(``acb_map_tc_batch``).  The reply of a request is the band map of its stream after that request --
the sum over the band's bins, as ``BeamformerBase.synthetic(f, num)`` returns it
(acoular/fbeamform.py:512-593) -- so each reply is the same whether the request was served alone or
in a mix.  Admission is bounded by an HBM budget: opening a stream or queueing a request that would
exceed it raises :class:`AdmissionError` (or waits, for requests, when ``block=True``).
"""

from __future__ import annotations

import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np
import torch

from . import device as D


class AdmissionError(RuntimeError):
    pass


@dataclass
class StreamState:
    sid: int
    mpos: torch.Tensor
    gpos: torch.Tensor
    gshape: tuple
    fs: float
    block_size: int
    window: str
    overlap: str
    bin_lo: int
    num_bins: int
    k: torch.Tensor
    steer_type: str
    r_diag: bool
    upper: torch.Tensor                 # running Welch sum, (num_bins, M, M) complex128
    tail: torch.Tensor                  # samples of the incomplete window
    csm: torch.Tensor = None            # finished CSM of the band's bins (num_bins, M, M) complex128
    out: torch.Tensor = None            # map of the band's bins (num_bins, G) float64
    band: torch.Tensor = None           # band map (G,) float64
    h_band: torch.Tensor = None         # pinned host copy of ``band``
    h_in: torch.Tensor = None           # pinned host staging of a request's samples (capacity, M) float32
    total_samples: int = 0
    bytes: int = 0
    gkey: object = None


@dataclass
class _Req:
    stream: StreamState
    samples: np.ndarray
    future: Future
    t_submit: float
    bytes: int
    t_done: float = 0.0
    extra: dict = field(default_factory=dict)


class BeamformingServer:
    def __init__(self, hbm_budget_bytes: int = 120 << 30, max_batch: int = 64, tc_precision: str = 'bf16x3',
                 device=None):
        self.dev = D.require_cuda(device)
        self.budget = int(hbm_budget_bytes)
        self.max_batch = max_batch
        self.tc_precision = tc_precision
        self.streams: dict[int, StreamState] = {}
        self._geom: dict = {}
        self._pending: list[_Req] = []
        self._cv = threading.Condition()
        self._used = 0
        self._stop = False
        self.batches: list[int] = []        # batch sizes served (for inspection)
        # per batch: (requests, t_taken, t_csm_issued, t_maps_issued, t_done), perf_counter seconds
        self.batch_times: list[tuple] = []
        self._err = torch.zeros(1, dtype=torch.int32, device=self.dev)     # kernel wait-timeout flag
        self._h_err = torch.zeros(1, dtype=torch.int32, pin_memory=True)
        self._worker = threading.Thread(target=self._run, name='acb-serving', daemon=True)
        self._worker.start()

    # ---------------------------------------------------------------- streams and admission
    def _reserve(self, nbytes: int, block: bool):
        with self._cv:
            while self._used + nbytes > self.budget:
                if not block or self._stop:
                    msg = f'HBM budget exceeded: {self._used + nbytes} > {self.budget} bytes'
                    raise AdmissionError(msg)
                self._cv.wait(timeout=0.05)
            self._used += nbytes

    def _release(self, nbytes: int):
        with self._cv:
            self._used -= nbytes
            self._cv.notify_all()

    @property
    def hbm_in_use(self) -> int:
        return self._used

    def open_stream(self, sid: int, mpos: np.ndarray, gpos: np.ndarray, sample_freq: float, block_size: int,
                    band: tuple, window: str = 'Hanning', overlap: str = '50%', steer_type: str = 'true level',
                    r_diag: bool = True, c: float = 343.0, gshape=None) -> StreamState:
        """Register a stream; ``band`` = (center frequency, 1/n octave) as in ``synthetic``."""
        freqs = np.abs(np.fft.fftfreq(block_size, 1.0 / sample_freq)[: block_size // 2 + 1])
        f, num = band
        f1, f2 = f * 2.0 ** (-0.5 / num), f * 2.0 ** (0.5 / num)
        i1, i2 = int(np.searchsorted(freqs, f1)), int(np.searchsorted(freqs, f2))
        if i1 == i2:
            msg = f'band ({f1:g} to {f2:g} Hz) contains no FFT line at block size {block_size}'
            raise ValueError(msg)
        M = mpos.shape[1]
        G = gpos.shape[1]
        nb = i2 - i1
        gkey = (mpos.tobytes(), gpos.tobytes())
        state_bytes = 2 * nb * M * M * 16 + block_size * M * 8 + nb * G * 8 + G * 8
        geo_bytes = 0 if gkey in self._geom else (mpos.size + gpos.size) * 8
        self._reserve(state_bytes + geo_bytes, block=False)
        if gkey not in self._geom:
            self._geom[gkey] = [torch.as_tensor(np.ascontiguousarray(mpos, dtype=np.float64), device=self.dev),
                                torch.as_tensor(np.ascontiguousarray(gpos, dtype=np.float64), device=self.dev), 0,
                                geo_bytes]
        self._geom[gkey][2] += 1            # streams sharing this geometry
        mp, gp = self._geom[gkey][0], self._geom[gkey][1]
        st = StreamState(sid=sid, mpos=mp, gpos=gp, gshape=gshape or (G,), fs=sample_freq, block_size=block_size,
                         window=window, overlap=overlap, bin_lo=i1, num_bins=nb,
                         k=torch.as_tensor(2 * np.pi * freqs[i1:i2] / c, dtype=torch.float64, device=self.dev),
                         steer_type=steer_type, r_diag=r_diag,
                         upper=torch.zeros((nb, M, M), dtype=torch.complex128, device=self.dev),
                         tail=torch.zeros((0, M), dtype=torch.float32, device=self.dev), bytes=state_bytes,
                         gkey=gkey,
                         csm=torch.empty((nb, M, M), dtype=torch.complex128, device=self.dev),
                         out=torch.empty((nb, G), dtype=torch.float64, device=self.dev),
                         band=torch.empty(G, dtype=torch.float64, device=self.dev),
                         h_band=torch.empty(G, dtype=torch.float64, pin_memory=True),
                         h_in=torch.empty((int(sample_freq * 0.25), M), dtype=torch.float32, pin_memory=True))
        self.streams[sid] = st
        return st

    def close_stream(self, sid: int):
        st = self.streams.pop(sid)
        self._release(st.bytes)
        g = self._geom[st.gkey]
        g[2] -= 1
        if g[2] == 0:                       # last stream on this geometry: free it
            del self._geom[st.gkey]
            self._release(g[3])

    def submit(self, sid: int, samples: np.ndarray, block: bool = True) -> Future:
        """Queue a block of samples (S, M) for stream ``sid``; the future yields the band map."""
        st = self.streams[sid]
        M = st.mpos.shape[1]
        G = st.gpos.shape[1]
        nb = st.num_bins
        from . import _native as N
        req_bytes = samples.size * 4 + nb * M * M * 16 + nb * G * 8 + \
            N.lib().acb_map_tc_workspace_bytes(M, nb, N.TC_PRECISIONS[self.tc_precision]) + \
            nb * M * max(1, samples.shape[0] // max(1, st.block_size // D.OVERLAPS[st.overlap])) * 16
        self._reserve(req_bytes, block=block)
        fut = Future()
        r = _Req(stream=st, samples=np.ascontiguousarray(samples, dtype=np.float32), future=fut,
                 t_submit=time.perf_counter(), bytes=req_bytes)
        with self._cv:
            self._pending.append(r)
            self._cv.notify_all()
        return fut

    # ---------------------------------------------------------------- worker
    def _take_batch(self):
        with self._cv:
            while not self._pending and not self._stop:
                self._cv.wait(timeout=0.05)
            if self._stop and not self._pending:
                return None
            # a stream's requests must be applied in order: at most one request per stream per batch
            batch, rest, seen = [], [], set()
            for r in self._pending:
                if r.stream.sid in seen or len(batch) >= self.max_batch:
                    rest.append(r)
                else:
                    seen.add(r.stream.sid)
                    batch.append(r)
            self._pending = rest
            return batch

    def _process(self, batch):
        dev = self.dev
        t_taken = time.perf_counter()
        insts = []
        for r in batch:
            st = r.stream
            S = r.samples.shape[0]
            if S > st.h_in.shape[0]:        # a request longer than any before on this stream
                st.h_in = torch.empty((S, st.h_in.shape[1]), dtype=torch.float32, pin_memory=True)
            st.h_in[:S].numpy()[...] = r.samples
            x = st.h_in[:S].to(dev, non_blocking=True)
            buf = torch.cat([st.tail, x], 0) if st.tail.shape[0] else x
            ov = D.OVERLAPS[st.overlap]
            hop = st.block_size // ov
            K = D.num_windows(buf.shape[0], st.block_size, ov)
            if K > 0:
                D.csm_upper_accumulate(buf.contiguous(), st.block_size, st.window, st.overlap, 'complex128',
                                       bin_lo=st.bin_lo, num_bins=st.num_bins, csm_upper=st.upper)
            st.tail = buf[K * hop:].clone()
            st.total_samples += r.samples.shape[0]
            _, weight = D.window_vector(st.window, st.block_size, dev)
            with np.errstate(divide='ignore', invalid='ignore'):
                scale = float(np.float64(2.0 / st.block_size) / np.float64(weight) /
                              np.float64(D.num_blocks(st.total_samples, st.block_size, ov)))
            D.csm_finalize(st.upper, scale, out=st.csm)
            M = st.mpos.shape[1]
            norm = (M / (M - 1.0)) if st.r_diag else 1.0
            insts.append(D.MapInstance(st.csm, st.k, st.mpos, st.gpos, st.steer_type, st.r_diag, norm,
                                       clip_negative=st.r_diag, out=st.out))
        t_csm = time.perf_counter()
        groups = {}
        for mi in insts:
            groups.setdefault(mi.steer_type, []).append(mi)
        for g in groups.values():
            for s0 in range(0, len(g), 64):
                D.map_tc_batch(g[s0:s0 + 64], precision=self.tc_precision, error_word=self._err)
        for r in batch:
            st = r.stream
            torch.sum(st.out, 0, out=st.band)
            st.h_band.copy_(st.band, non_blocking=True)
        self._h_err.copy_(self._err, non_blocking=True)
        t_maps = time.perf_counter()
        torch.cuda.current_stream(dev).synchronize()
        now = time.perf_counter()
        self.batch_times.append((len(batch), t_taken, t_csm, t_maps, now))
        if int(self._h_err[0]):
            self._err.zero_()
            msg = 'acb_map_tc_batch: a tensor-core pipeline wait timed out'
            raise RuntimeError(msg)
        for r in batch:
            r.t_done = now
            r.future.latency = now - r.t_submit     # submit -> result ready, seconds
            r.future.units = r.stream.out.numel()   # grid points x bins mapped for this request
            r.future.set_result(r.stream.h_band.numpy().reshape(r.stream.gshape).copy())
        self.batches.append(len(batch))

    def _run(self):
        torch.cuda.set_device(self.dev)
        while True:
            batch = self._take_batch()
            if batch is None:
                return
            try:
                self._process(batch)
            except Exception as e:  # noqa: BLE001 - every waiting caller gets the error
                for r in batch:
                    if not r.future.done():
                        r.future.set_exception(e)
            finally:
                for r in batch:
                    self._release(r.bytes)

    def close(self):
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        self._worker.join(timeout=30)
