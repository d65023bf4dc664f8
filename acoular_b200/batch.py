"""Batched beamforming of many uneven instances on one GPU.

An instance is one array recording with its own geometry, grid, FFT block size and bin range --
the unit ``PowerSpectra`` + ``BeamformerBase`` process in the reference (acoular/spectra.py:366-416,
acoular/fbeamform.py:475-510).  :class:`BatchPlan` keeps every instance's buffers resident and runs

1. per instance: the windowed FFT + Welch accumulation for the instance's bins only
   (``acb_csm_accumulate``) and the Hermitian finish (``acb_csm_finalize``);
2. one persistent tensor-core launch for the maps of all instances (``acb_map_tc_batch``; up to 64
   instances per launch, one launch per steering type).

The whole sequence can be captured once in a CUDA graph (``capture()``) and replayed for new data
(``load_samples`` + ``run``): the launch list is then a single graph launch.  Each instance's map is
bit-identical to what the same instance gives alone (the map kernel computes each item
independently of what shares the launch).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N
from . import device as D


@dataclass
class Instance:
    """Inputs of one instance.  ``samples``: (S, M) float32/float64 (host or device)."""

    samples: object
    mpos: np.ndarray            # (3, M)
    gpos: np.ndarray            # (3, G)
    sample_freq: float
    block_size: int
    bin_lo: int
    num_bins: int
    window: str = 'Hanning'
    overlap: str = '50%'
    precision: str = 'complex64'
    steer_type: str = 'true level'
    r_diag: bool = True
    r_diag_norm: float = 0.0
    c: float = 343.0
    ref: object = None


class BatchPlan:
    """Resident buffers and launches for a fixed list of instances."""

    def __init__(self, instances, form: str = 'tc', tc_precision: str = 'bf16x3', device=None):
        self.dev = D.require_cuda(device)
        self.form = form
        self.tc_precision = tc_precision
        self.inst = list(instances)
        self.graph = None
        dev = self.dev
        self.samples, self.upper, self.csm, self.k, self.mpos, self.gpos, self.out = [], [], [], [], [], [], []
        self.scale, self.windows, self.norm = [], [], []
        ws_bytes = 0
        for it in self.inst:
            S, M = np.shape(it.samples)
            if isinstance(it.samples, torch.Tensor):
                dtype = torch.float32 if it.samples.dtype == torch.float32 else torch.float64
            else:
                dtype = torch.float32 if np.asarray(it.samples).dtype == np.float32 else torch.float64
            self.samples.append(torch.empty((S, M), dtype=dtype, device=dev))
            cdt = torch.complex64 if it.precision == 'complex64' else torch.complex128
            self.upper.append(torch.zeros((it.num_bins, M, M), dtype=cdt, device=dev))
            self.csm.append(torch.empty((it.num_bins, M, M), dtype=torch.complex128, device=dev))
            freqs = np.abs(np.fft.fftfreq(it.block_size, 1.0 / it.sample_freq)[: it.block_size // 2 + 1])
            bins = np.arange(it.bin_lo, it.bin_lo + it.num_bins)
            self.k.append(torch.as_tensor(2 * np.pi * freqs[bins] / it.c, dtype=torch.float64, device=dev))
            self.mpos.append(torch.as_tensor(np.ascontiguousarray(it.mpos, dtype=np.float64), device=dev))
            self.gpos.append(torch.as_tensor(np.ascontiguousarray(it.gpos, dtype=np.float64), device=dev))
            self.out.append(torch.empty((it.num_bins, it.gpos.shape[1]), dtype=torch.float64, device=dev))
            ov = D.OVERLAPS[it.overlap]
            K = D.num_windows(S, it.block_size, ov)
            self.windows.append(K)
            _, weight = D.window_vector(it.window, it.block_size, dev)
            with np.errstate(divide='ignore', invalid='ignore'):
                self.scale.append(float(np.float64(2.0 / it.block_size) / np.float64(weight) /
                                        np.float64(D.num_blocks(S, it.block_size, ov))))
            prec = N.C64 if it.precision == 'complex64' else N.C128
            ws_bytes = max(ws_bytes, N.lib().acb_csm_workspace_bytes_block(M, it.num_bins, max(K, 1), prec,
                                                                             it.block_size))
            if it.r_diag:
                self.norm.append(it.r_diag_norm if it.r_diag_norm != 0.0 else M / (M - 1.0))
            else:
                self.norm.append(1.0)
        self.csm_ws = torch.empty(max(ws_bytes, 16), dtype=torch.uint8, device=dev)
        self.load_samples([it.samples for it in self.inst])
        self.map_instances = [
            D.MapInstance(self.csm[i], self.k[i], self.mpos[i], self.gpos[i], it.steer_type, it.r_diag,
                          self.norm[i], ref=it.ref, clip_negative=it.r_diag, out=self.out[i])
            for i, it in enumerate(self.inst)]
        self.error_word = torch.zeros(1, dtype=torch.int32, device=dev)

    def load_samples(self, samples_list):
        """Copy new sample arrays (same shapes) into the resident buffers."""
        for buf, x in zip(self.samples, samples_list):
            t = x if isinstance(x, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(x))
            buf.copy_(t.to(buf.dtype), non_blocking=t.device.type == 'cpu' and t.is_pinned())

    def _launch(self):
        for i, it in enumerate(self.inst):
            self.upper[i].zero_()
            D.csm_upper_accumulate(self.samples[i], it.block_size, it.window, it.overlap, it.precision,
                                   bin_lo=it.bin_lo, num_bins=it.num_bins, csm_upper=self.upper[i],
                                   workspace=self.csm_ws, max_workspace_bytes=self.csm_ws.numel())
            D.csm_finalize(self.upper[i], self.scale[i], out=self.csm[i])
        if self.form == 'tc':
            groups = {}
            for mi in self.map_instances:
                groups.setdefault(mi.steer_type, []).append(mi)
            for g in groups.values():
                for s0 in range(0, len(g), 64):
                    D.map_tc_batch(g[s0:s0 + 64], precision=self.tc_precision, error_word=self.error_word)
        else:
            for mi in self.map_instances:
                D.map_f64(mi.csm, mi.wavenumbers, mi.mpos, mi.gpos, mi.steer_type, mi.r_diag, mi.norm, ref=mi.ref,
                          clip_negative=mi.clip_negative, out=mi.out)

    def capture(self):
        """Capture the whole batch (CSMs + maps) in one CUDA graph."""
        self._launch()                      # warm-up: workspaces and kernel attributes outside capture
        torch.cuda.synchronize(self.dev)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._launch()
        self.graph = g
        return self

    def run(self):
        """Compute every instance's maps (graph replay if captured); returns the device outputs."""
        if self.graph is not None:
            self.graph.replay()
        else:
            self._launch()
        return self.out

    def units(self) -> int:
        """grid-pts x bins of one run."""
        return int(sum(it.gpos.shape[1] * it.num_bins for it in self.inst))
