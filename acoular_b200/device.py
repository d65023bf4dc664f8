"""Device-level entry points: resident buffers, CSM and map launches on the current torch stream.

Everything here takes and returns torch CUDA tensors; the Acoular-compatible classes in
:mod:`acoular_b200.spectra` and :mod:`acoular_b200.fbeamform` wrap these for numpy users.
"""

from __future__ import annotations

import ctypes
import hashlib
import os
import threading
from pathlib import Path

import numpy as np
import torch

from . import _native as N

WINDOWS = {
    'Rectangular': np.ones,
    'Hanning': np.hanning,
    'Hamming': np.hamming,
    'Bartlett': np.bartlett,
    'Blackman': np.blackman,
}
OVERLAPS = {'None': 1, '50%': 2, '75%': 4, '87.5%': 8}

DEFAULT_WORKSPACE_BYTES = 2 << 30


def require_cuda(device=None) -> torch.device:
    if not torch.cuda.is_available():
        msg = 'acoular_b200 needs a CUDA device (B200, sm_100a); no CPU fallback exists'
        raise RuntimeError(msg)
    N.lib()
    return torch.device('cuda', torch.cuda.current_device() if device is None else torch.device(device).index or 0)


def num_windows(num_samples: int, block_size: int, overlap: int) -> int:
    """Windows yielded by ``_get_source_data`` (acoular/spectra.py:171-184): starts j*hop with
    j*hop + block_size <= num_samples."""
    hop = block_size // overlap
    if num_samples < block_size:
        return 0
    return (num_samples - block_size) // hop + 1


def num_blocks(num_samples: int, block_size: int, overlap: int) -> float:
    """The reference's averaging divisor (acoular/spectra.py:281-283), a float formula."""
    return overlap * num_samples / block_size - overlap + 1


_tw_cache: dict = {}
_win_cache: dict = {}


def twiddles(block_size: int, device) -> torch.Tensor:
    key = (block_size, str(device))
    t = _tw_cache.get(key)
    if t is None:
        k = np.arange(block_size // 2)
        w = np.exp(-2j * np.pi * k / block_size)
        t = torch.as_tensor(w.astype(np.complex128), device=device)
        _tw_cache[key] = t
    return t


def window_vector(window: str, block_size: int, device) -> tuple[torch.Tensor, float]:
    key = (window, block_size, str(device))
    v = _win_cache.get(key)
    if v is None:
        w = WINDOWS[window](block_size).astype(np.float64)
        v = (torch.as_tensor(w, device=device), float(np.dot(w, w)))
        _win_cache[key] = v
    return v


CSM_PRECISIONS = {'complex128': N.C128, 'complex64': N.C64, 'tc_tf32': N.CSM_TC_TF32, 'tc_bf16x3': N.CSM_TC_BF16X3}


def csm_upper_accumulate(samples: torch.Tensor, block_size: int, window: str, overlap: str,
                         precision: str = 'complex128', bin_lo: int = 0, num_bins: int | None = None,
                         csm_upper: torch.Tensor | None = None, workspace: torch.Tensor | None = None,
                         max_workspace_bytes: int = DEFAULT_WORKSPACE_BYTES, first_window: int = 0,
                         windows: int | None = None):
    """Welch sum (upper triangle) of all windows of ``samples`` (device, (S, M) f32/f64).

    ``precision``: ``'complex128'`` / ``'complex64'`` (the reference's CSM precisions, FP64 / FP32
    Gram in the reference's accumulation order) or ``'tc_tf32'`` / ``'tc_bf16x3'`` (the tensor-core
    Gram: TF32 or split-BF16 operands, FP32 accumulation per chunk of windows, complex128 sums).
    Returns ``(csm_upper, n_windows)``; ``csm_upper`` is (num_bins, M, M) complex128/complex64.
    """
    dev = samples.device
    if samples.dim() != 2 or not samples.is_contiguous():
        msg = 'samples must be a contiguous (num_samples, num_mics) tensor'
        raise ValueError(msg)
    S, M = samples.shape
    ov = OVERLAPS[overlap]
    hop = block_size // ov
    F = block_size // 2 + 1
    nb = F - bin_lo if num_bins is None else num_bins
    prec = CSM_PRECISIONS[precision]
    cdt = torch.complex64 if prec == N.C64 else torch.complex128
    if csm_upper is None:
        csm_upper = torch.zeros((nb, M, M), dtype=cdt, device=dev)
    K = num_windows(S, block_size, ov) if windows is None else windows
    sd = N.F32 if samples.dtype == torch.float32 else N.F64
    if samples.dtype not in (torch.float32, torch.float64):
        samples = samples.to(torch.float64)
        sd = N.F64
    wv, _ = window_vector(window, block_size, dev)
    tw = twiddles(block_size, dev)
    if prec in (N.CSM_TC_TF32, N.CSM_TC_BF16X3):
        # the tensor-core operand pads every chunk to whole blocks of 32 windows
        per32 = N.lib().acb_csm_workspace_bytes_block(M, nb, 32, prec, block_size)
        chunk = int(max(32, min(65504, max_workspace_bytes // max(per32, 1) * 32)))
        chunk = min(chunk, -(-max(K, 1) // 32) * 32)
        need = N.lib().acb_csm_workspace_bytes_block(M, nb, chunk, prec, block_size)
    else:
        per_win = N.lib().acb_csm_workspace_bytes_block(M, nb, 1, prec, block_size)
        chunk = int(max(1, min(65535, max_workspace_bytes // max(per_win, 1), K if K > 0 else 1)))
        need = N.lib().acb_csm_workspace_bytes_block(M, nb, chunk, prec, block_size)
    if workspace is None or workspace.numel() < need:
        workspace = torch.empty(need, dtype=torch.uint8, device=dev)
    st = N.stream_handle()
    L = N.lib()
    w = first_window
    end = first_window + K
    while w < end:
        nw = min(chunk, end - w)
        N.check(L.acb_csm_accumulate(samples.data_ptr(), sd, S, M, block_size, hop, w, nw, wv.data_ptr(),
                                     tw.data_ptr(), bin_lo, nb, prec, csm_upper.data_ptr(), workspace.data_ptr(),
                                     workspace.numel(), st), 'acb_csm_accumulate')
        w += nw
    return csm_upper, K


_copy_streams: dict = {}


def copy_stream(device) -> torch.cuda.Stream:
    """A side stream per device for host<->device copies that overlap the computation."""
    key = str(device)
    s = _copy_streams.get(key)
    if s is None:
        s = torch.cuda.Stream(device=device)
        _copy_streams[key] = s
    return s


def csm_finalize(csm_upper: torch.Tensor, scale: float, out: torch.Tensor | None = None) -> torch.Tensor:
    nb, M, _ = csm_upper.shape
    prec = N.C64 if csm_upper.dtype == torch.complex64 else N.C128
    if out is None:
        out = torch.empty((nb, M, M), dtype=torch.complex128, device=csm_upper.device)
    N.check(N.lib().acb_csm_finalize(csm_upper.data_ptr(), nb, M, prec, float(scale), out.data_ptr(),
                                     N.stream_handle()), 'acb_csm_finalize')
    return out


def calc_csm(samples: torch.Tensor, block_size: int = 1024, window: str = 'Rectangular', overlap: str = 'None',
             precision: str = 'complex128', bin_lo: int = 0, num_bins: int | None = None,
             max_workspace_bytes: int = DEFAULT_WORKSPACE_BYTES) -> torch.Tensor:
    """Full CSM (num_bins, M, M) complex128 on the device, as ``PowerSpectra.calc_csm`` returns it."""
    ov = OVERLAPS[overlap]
    up, _ = csm_upper_accumulate(samples, block_size, window, overlap, precision, bin_lo, num_bins,
                                 max_workspace_bytes=max_workspace_bytes)
    _, weight = window_vector(window, block_size, samples.device)
    nblk = num_blocks(samples.shape[0], block_size, ov)
    with np.errstate(divide='ignore', invalid='ignore'):
        scale = np.float64(2.0 / block_size) / np.float64(weight) / np.float64(nblk)
    return csm_finalize(up, float(scale))


# ------------------------------------------------------------------------------------------------
# sincos exception table (glibc-faithful plain form)
# ------------------------------------------------------------------------------------------------
SINCOS_MAX_ARG = 2048.0
SINCOS_SLOTS = 1 << 23
_table_lock = threading.Lock()
_table_host = None
_table_dev: dict = {}


def _cache_dir() -> Path:
    d = Path(os.environ.get('ACOULAR_B200_CACHE', Path.home() / '.cache' / 'acoular_b200'))
    d.mkdir(parents=True, exist_ok=True)
    return d


def sincos_table_host() -> np.ndarray:
    """Exception table of the host C library's float32 cosf/sinf over [0, 2048) (built once, cached)."""
    global _table_host
    with _table_lock:
        if _table_host is not None:
            return _table_host
        libc_ver = os.confstr('CS_GNU_LIBC_VERSION') if hasattr(os, 'confstr') else 'unknown'
        tag = hashlib.blake2b(f'{libc_ver}|{SINCOS_MAX_ARG}|{SINCOS_SLOTS}|v1'.encode(), digest_size=8).hexdigest()
        path = _cache_dir() / f'sincos_exc_{tag}.npy'
        if path.exists():
            try:
                _table_host = np.load(path)
                return _table_host
            except Exception:  # noqa: BLE001 - rebuild a corrupt cache file
                pass
        tab = np.empty(SINCOS_SLOTS, dtype=np.uint64)
        n = N.lib().acb_sincos_table_build_host(tab.ctypes.data_as(ctypes.c_void_p), SINCOS_SLOTS,
                                                ctypes.c_float(SINCOS_MAX_ARG), N.nproc())
        if n < 0:
            raise N.AcbError(int(-n), 'acb_sincos_table_build_host')
        tmp = path.with_suffix(f'.{os.getpid()}.tmp.npy')
        np.save(tmp, tab)
        os.replace(tmp, path)
        _table_host = tab
        return tab


def sincos_table_device(device) -> torch.Tensor:
    key = str(device)
    t = _table_dev.get(key)
    if t is None:
        t = torch.as_tensor(sincos_table_host().view(np.int64), device=device)
        _table_dev[key] = t
    return t


# ------------------------------------------------------------------------------------------------
# map
# ------------------------------------------------------------------------------------------------
def map_params(num_mics, num_grid, num_bins, steer_type, r_diag, norm, clip_negative=None, ref=None,
               glibc_faithful=False, device=None, tc_pass_chunks: int = 0, tc_splits: int = 0) -> N.MapParams:
    p = N.MapParams()
    p.tc_pass_chunks = int(tc_pass_chunks)
    p.tc_splits = int(tc_splits)
    p.num_mics = int(num_mics)
    p.num_grid = int(num_grid)
    p.num_bins = int(num_bins)
    p.steer_type = N.STEER_CODES[steer_type]
    p.r_diag = int(bool(r_diag))
    p.clip_negative = int(bool(r_diag) if clip_negative is None else bool(clip_negative))
    p.norm = float(norm)
    if ref is None:
        p.ref_mode = 0
        p.ref_point[:] = (0.0, 0.0, 0.0)
    elif np.isscalar(ref):
        if float(ref) > 0:
            p.ref_mode = 1
            p.ref_distance = float(ref)
        else:
            p.ref_mode = 0
            p.ref_point[:] = (0.0, 0.0, 0.0)
    else:
        p.ref_mode = 0
        p.ref_point[:] = tuple(float(x) for x in np.asarray(ref, dtype=float).reshape(3))
    if glibc_faithful:
        t = sincos_table_device(device)
        p.glibc_faithful = 1
        p.sincos_table = t.data_ptr()
        p.sincos_table_slots = t.numel()
    return p


def map_f64(csm: torch.Tensor, wavenumbers: torch.Tensor, mpos: torch.Tensor, gpos: torch.Tensor, steer_type: str,
            r_diag: bool, norm: float, ref=None, clip_negative=None, glibc_faithful=True,
            out: torch.Tensor | None = None, steer_norm: torch.Tensor | None = None) -> torch.Tensor:
    """Plain FP64 map for B bins: csm (B, M, M) complex128, wavenumbers (B,) -> (B, G) float64."""
    B, M, _ = csm.shape
    G = gpos.shape[1]
    dev = csm.device
    p = map_params(M, G, B, steer_type, r_diag, norm, clip_negative, ref, glibc_faithful, dev)
    if out is None:
        out = torch.empty((B, G), dtype=torch.float64, device=dev)
    N.check(N.lib().acb_map_f64(ctypes.byref(p), csm.data_ptr(), wavenumbers.data_ptr(), mpos.data_ptr(),
                                gpos.data_ptr(), out.data_ptr(), N.ptr(steer_norm), None, N.stream_handle()),
            'acb_map_f64')
    return out


def map_eig_f64(eigval: torch.Tensor, eigvec: torch.Tensor, wavenumbers: torch.Tensor, mpos: torch.Tensor,
                gpos: torch.Tensor, steer_type: str, r_diag: bool, norm: float, ref=None, clip_negative=None,
                glibc_faithful=True, out: torch.Tensor | None = None,
                steer_norm: torch.Tensor | None = None) -> torch.Tensor:
    """Eigenvalue form of the plain FP64 map for B bins: eigval (B, E) float64, eigvec (B, M, E)
    complex128 (columns = eigenvectors), wavenumbers (B,) -> (B, G) float64."""
    B, M, E = eigvec.shape
    if tuple(eigval.shape) != (B, E):
        msg = 'eigval must be (num_bins, num_eigs) and eigvec (num_bins, num_mics, num_eigs)'
        raise ValueError(msg)
    if not (eigval.is_contiguous() and eigvec.is_contiguous()):
        msg = 'eigval and eigvec must be contiguous'
        raise ValueError(msg)
    G = gpos.shape[1]
    dev = eigvec.device
    p = map_params(M, G, B, steer_type, r_diag, norm, clip_negative, ref, glibc_faithful, dev)
    if out is None:
        out = torch.empty((B, G), dtype=torch.float64, device=dev)
    N.check(N.lib().acb_map_eig_f64(ctypes.byref(p), E, eigval.data_ptr(), eigvec.data_ptr(), wavenumbers.data_ptr(),
                                    mpos.data_ptr(), gpos.data_ptr(), out.data_ptr(), N.ptr(steer_norm),
                                    N.stream_handle()), 'acb_map_eig_f64')
    return out


def map_rm_f64(csm: torch.Tensor, wavenumbers: torch.Tensor, r0: torch.Tensor, rm: torch.Tensor, steer_type: str,
               r_diag: bool, norm: float, clip_negative=None, glibc_faithful=True, out: torch.Tensor | None = None,
               steer_norm: torch.Tensor | None = None) -> torch.Tensor:
    """Plain FP64 map with given distances r0 (G,), rm (G, M) (any environment) for B bins."""
    B, M, _ = csm.shape
    G = rm.shape[0]
    dev = csm.device
    p = map_params(M, G, B, steer_type, r_diag, norm, clip_negative, None, glibc_faithful, dev)
    if out is None:
        out = torch.empty((B, G), dtype=torch.float64, device=dev)
    N.check(N.lib().acb_map_rm_f64(ctypes.byref(p), csm.data_ptr(), wavenumbers.data_ptr(), r0.data_ptr(),
                                   rm.data_ptr(), out.data_ptr(), N.ptr(steer_norm), N.stream_handle()),
            'acb_map_rm_f64')
    return out


def map_custom_f64(csm: torch.Tensor, steer: torch.Tensor, r_diag: bool, norm: float, clip_negative=False,
                   out: torch.Tensor | None = None, steer_norm: torch.Tensor | None = None,
                   eig: tuple | None = None) -> torch.Tensor:
    """Map with custom steering vectors steer (B, G, M) complex128 for B bins; with ``eig`` =
    (eigval (B, E), eigvec (B, M, E)) the eigenvalue form (``csm`` unused)."""
    B, G, M = steer.shape
    dev = steer.device
    if not steer.is_contiguous():
        msg = 'steer must be a contiguous (num_bins, num_grid, num_mics) complex128 tensor'
        raise ValueError(msg)
    p = map_params(M, G, B, 'classic', r_diag, norm, clip_negative, None, False, dev)
    if out is None:
        out = torch.empty((B, G), dtype=torch.float64, device=dev)
    if eig is None:
        N.check(N.lib().acb_map_custom_f64(ctypes.byref(p), csm.data_ptr(), steer.data_ptr(), out.data_ptr(),
                                           N.ptr(steer_norm), N.stream_handle()), 'acb_map_custom_f64')
    else:
        ev, evec = eig
        N.check(N.lib().acb_map_eig_custom_f64(ctypes.byref(p), ev.shape[1], ev.data_ptr(), evec.data_ptr(),
                                               steer.data_ptr(), out.data_ptr(), N.ptr(steer_norm),
                                               N.stream_handle()), 'acb_map_eig_custom_f64')
    return out


def map_eig_rm_f64(eigval: torch.Tensor, eigvec: torch.Tensor, k: float, r0: torch.Tensor, rm: torch.Tensor,
                   steer_type: str, r_diag: bool, norm: float, glibc_faithful=True, out: torch.Tensor | None = None,
                   steer_norm: torch.Tensor | None = None) -> torch.Tensor:
    """Eigenvalue form for one bin with given distances r0 (G,), rm (G, M): eigval (1, E), eigvec (1, M, E)."""
    _, M, E = eigvec.shape
    G = rm.shape[0]
    dev = eigvec.device
    p = map_params(M, G, 1, steer_type, r_diag, norm, False, None, glibc_faithful, dev)
    if out is None:
        out = torch.empty(G, dtype=torch.float64, device=dev)
    N.check(N.lib().acb_beamformer_freq_eig_f64(ctypes.byref(p), E, eigval.data_ptr(), eigvec.data_ptr(), float(k),
                                                r0.data_ptr(), rm.data_ptr(), out.data_ptr(), N.ptr(steer_norm),
                                                N.stream_handle()), 'acb_beamformer_freq_eig_f64')
    return out


_tc_ws: dict = {}


def map_tc_workspace(num_mics: int, num_bins: int, precision: str, device) -> torch.Tensor:
    """Cached scratch buffer for the split-BF16 copy of the real-embedded CSM."""
    need = N.lib().acb_map_tc_workspace_bytes(num_mics, num_bins, N.TC_PRECISIONS[precision])
    key = str(device)
    ws = _tc_ws.get(key)
    if ws is None or ws.numel() < need:
        ws = torch.empty(need, dtype=torch.uint8, device=device)
        _tc_ws[key] = ws
    return ws


def map_tc(csm: torch.Tensor, wavenumbers: torch.Tensor, mpos: torch.Tensor, gpos: torch.Tensor, steer_type: str,
           r_diag: bool, norm: float, ref=None, clip_negative=None, precision: str = 'bf16x3',
           out: torch.Tensor | None = None, steer_norm: torch.Tensor | None = None,
           error_word: torch.Tensor | None = None, tuning='auto') -> torch.Tensor:
    """Tensor-core map for B bins (same contract as :func:`map_f64`).

    ``tuning``: ``'auto'`` (the autotuned (pass width, split) of this shape class, through the batch
    entry, so the result equals the one the same instance gets inside any batch), ``None`` (the
    single-instance entry ``acb_map_tc`` with the default tile and no split), or an explicit
    ``(pass_chunks, splits)``.
    """
    if tuning is not None:
        mi = MapInstance(csm, wavenumbers, mpos, gpos, steer_type, r_diag, norm, ref=ref, clip_negative=clip_negative,
                         out=out, steer_norm=steer_norm, tuning=None if tuning == 'auto' else tuning)
        return map_tc_batch([mi], precision=precision, error_word=error_word)[0]
    B, M, _ = csm.shape
    G = gpos.shape[1]
    dev = csm.device
    p = map_params(M, G, B, steer_type, r_diag, norm, clip_negative, ref, False, dev)
    if out is None:
        out = torch.empty((B, G), dtype=torch.float64, device=dev)
    ws = map_tc_workspace(M, B, precision, dev)
    N.check(N.lib().acb_map_tc(ctypes.byref(p), N.TC_PRECISIONS[precision], csm.data_ptr(), wavenumbers.data_ptr(),
                               mpos.data_ptr(), gpos.data_ptr(), out.data_ptr(), N.ptr(steer_norm), ws.data_ptr(),
                               ws.numel(), N.ptr(error_word), N.stream_handle()), 'acb_map_tc')
    return out


class MapInstance:
    """One map of a batch: device tensors of its CSM (B, M, M) c128, wave numbers (B,), positions,
    the output (B, G) and the beamformer settings."""

    def __init__(self, csm, wavenumbers, mpos, gpos, steer_type='true level', r_diag=True, norm=1.0, ref=None,
                 clip_negative=None, out=None, steer_norm=None, tuning=None):
        self.tuning = tuning            # (pass_chunks, splits) or None: the autotuned value
        self.csm, self.wavenumbers, self.mpos, self.gpos = csm, wavenumbers, mpos, gpos
        self.steer_type, self.r_diag, self.norm, self.ref = steer_type, r_diag, norm, ref
        self.clip_negative = clip_negative
        B, M, _ = csm.shape
        self.out = out if out is not None else torch.empty((B, gpos.shape[1]), dtype=torch.float64,
                                                           device=csm.device)
        self.steer_norm = steer_norm


_batch_ws: dict = {}


def map_tc_batch(instances, precision: str = 'bf16x3', error_word: torch.Tensor | None = None):
    """Many maps of uneven shape in one persistent tensor-core launch (<= 64 per call, one steer type)."""
    if not instances:
        return []
    dev = instances[0].csm.device
    n = len(instances)
    params = (N.MapParams * n)()
    io = (N.MapIO * n)()
    from . import autotune
    for i, it in enumerate(instances):
        B, M, _ = it.csm.shape
        G = it.gpos.shape[1]
        pw, sp = it.tuning if it.tuning is not None else autotune.lookup(M, G, B, precision)
        params[i] = map_params(M, G, B, it.steer_type, it.r_diag, it.norm, it.clip_negative, it.ref,
                               False, dev, tc_pass_chunks=pw, tc_splits=sp)
        io[i].csm, io[i].wavenumber = it.csm.data_ptr(), it.wavenumbers.data_ptr()
        io[i].mpos, io[i].gpos = it.mpos.data_ptr(), it.gpos.data_ptr()
        io[i].out_map, io[i].out_steer_norm = it.out.data_ptr(), N.ptr(it.steer_norm)
    prec = N.TC_PRECISIONS[precision]
    need = N.lib().acb_map_tc_batch_workspace_bytes(params, n, prec)
    ws = _batch_ws.get(str(dev))
    if ws is None or ws.numel() < need:
        ws = torch.empty(need, dtype=torch.uint8, device=dev)
        _batch_ws[str(dev)] = ws
    N.check(N.lib().acb_map_tc_batch(params, io, n, prec, ws.data_ptr(), ws.numel(), N.ptr(error_word),
                                     N.stream_handle()), 'acb_map_tc_batch')
    return [it.out for it in instances]


# ------------------------------------------------------------------------------------------------
# point-spread functions and DAMAS
# ------------------------------------------------------------------------------------------------
def psf_f64(r0: torch.Tensor, rm: torch.Tensor, k: float, sources: torch.Tensor, steer_type: str,
            round_f32: bool = False, glibc_faithful: bool = True, out: torch.Tensor | None = None) -> torch.Tensor:
    """PSF (G, S) of unit sources at the grid points ``sources`` (int64, (S,), a numpy array, checked
    here, or a device tensor, whose out-of-grid indices give NaN columns) for one wave number,
    distances r0 (G,), rm (G, M) float64 on the device (calcPointSpreadFunction)."""
    G, M = rm.shape
    if not (r0.is_contiguous() and rm.is_contiguous()) or r0.dtype != torch.float64 or rm.dtype != torch.float64:
        msg = 'r0 and rm must be contiguous float64 tensors'
        raise ValueError(msg)
    if isinstance(sources, np.ndarray):
        if sources.size and (sources.min() < 0 or sources.max() >= G):
            msg = f'source indices must lie in [0, {G})'
            raise IndexError(msg)
        sources = torch.as_tensor(sources)
    # indices of a device tensor are checked by the kernel: a column outside the grid is NaN
    sources = sources.to(device=rm.device, dtype=torch.int64).contiguous()
    S = sources.numel()
    p = map_params(M, G, 1, steer_type, False, 1.0, False, None, glibc_faithful, rm.device)
    if out is None:
        out = torch.empty((G, S), dtype=torch.float64, device=rm.device)
    if S == 0:
        return out
    N.check(N.lib().acb_psf_f64(ctypes.byref(p), S, sources.data_ptr(), float(k), r0.data_ptr(), rm.data_ptr(),
                                int(bool(round_f32)), out.data_ptr(), N.stream_handle()), 'acb_psf_f64')
    return out


def damas_gauss_seidel(psf: torch.Tensor, dirty_map: torch.Tensor, n_iter: int, relax: float,
                       solution: torch.Tensor | None = None, cta_per_bin: int = 0) -> torch.Tensor:
    """DAMAS Gauss-Seidel sweeps for B bins: psf (B, G, G), dirty_map (B, G) float64; ``solution``
    (B, G) holds the start (default: the dirty map) and receives the result."""
    B, G = dirty_map.shape
    if tuple(psf.shape) != (B, G, G):
        msg = f'psf must be (num_bins, num_grid, num_grid) = ({B}, {G}, {G}), got {tuple(psf.shape)}'
        raise ValueError(msg)
    for t in (psf, dirty_map):
        if t.dtype != torch.float64 or not t.is_contiguous():
            msg = 'psf and dirty_map must be contiguous float64 tensors'
            raise ValueError(msg)
    if solution is None:
        solution = dirty_map.clone()
    if B == 0 or G == 0:
        return solution
    N.check(N.lib().acb_damas_gauss_seidel_f64(psf.data_ptr(), G, B, dirty_map.data_ptr(), solution.data_ptr(),
                                               int(n_iter), float(relax), int(cta_per_bin), N.stream_handle()),
            'acb_damas_gauss_seidel_f64')
    return solution


# ------------------------------------------------------------------------------------------------
# CLEAN-SC
# ------------------------------------------------------------------------------------------------
def heevd_f64(csm: torch.Tensor, chunk_bytes: int = 4 << 30):
    """Hermitian eigendecomposition of every bin: csm (B, M, M) complex128 on the device ->
    (eigvals (B, M) float64 ascending, eigvecs (B, M, M) complex128, eigenvectors in the columns, info (B,)
    int32), the layout numpy.linalg.eigh returns; bins in chunks whose workspace fits ``chunk_bytes``."""
    B, M, _ = csm.shape
    dev = csm.device
    c = csm.to(torch.complex128).contiguous()
    ev = torch.empty((B, M), dtype=torch.float64, device=dev)
    vec = torch.empty((B, M, M), dtype=torch.complex128, device=dev)
    info = torch.zeros(B, dtype=torch.int32, device=dev)
    per = max(1, N.lib().acb_heevd_workspace_bytes(M, 1))
    step = int(max(1, min(B, chunk_bytes // per)))
    ws = torch.empty(N.lib().acb_heevd_workspace_bytes(M, step), dtype=torch.uint8, device=dev)
    for b0 in range(0, B, step):
        nb = min(step, B - b0)
        N.check(N.lib().acb_heevd_f64(c[b0].data_ptr(), nb, M, ev[b0].data_ptr(), vec[b0].data_ptr(),
                                      info[b0].data_ptr(), ws.data_ptr(), ws.numel(), N.stream_handle()),
                'acb_heevd_f64')
    return ev, vec, info


def heevd_select_supported(num_mics: int, num_ranks: int = 1) -> bool:
    """Whether acb_heevd_select_f64 takes this size: its per-matrix work arrays, (3 M + 5 M E) doubles and M E
    pivot flags, must fit 200 KB of shared memory (M up to about 3100 for one rank)."""
    M, E = int(num_mics), int(num_ranks)
    return 1 <= E <= 4 and E <= M <= 4096 and (3 * M + 5 * M * E) * 8 + M * E <= 200 * 1024


def heevd_select_f64(csm: torch.Tensor, ranks, chunk_bytes: int = 4 << 30):
    """Selected eigenpairs of every bin: csm (B, M, M) complex128 on the device, ``ranks`` (1 to 4 ascending
    ranks, the same for every bin; -1 is the largest) -> (eigvals (B, E) float64, eigvecs (B, M, E)
    complex128), as the columns ``ranks`` of :func:`heevd_f64`'s result (up to a unit phase per column)."""
    B, M, _ = csm.shape
    dev = csm.device
    sel = [int(r) % M for r in ranks]
    E = len(sel)
    if not 1 <= E <= 4:
        msg = 'between 1 and 4 ranks'
        raise ValueError(msg)
    c = csm.to(torch.complex128).contiguous()
    ev = torch.empty((B, E), dtype=torch.float64, device=dev)
    vec = torch.empty((B, M, E), dtype=torch.complex128, device=dev)
    sel_h = (ctypes.c_int * E)(*sel)
    per = max(1, N.lib().acb_heevd_workspace_bytes(M, 1))
    step = int(max(1, min(B, chunk_bytes // per)))
    ws = torch.empty(N.lib().acb_heevd_workspace_bytes(M, step), dtype=torch.uint8, device=dev)
    for b0 in range(0, B, step):
        nb = min(step, B - b0)
        N.check(N.lib().acb_heevd_select_f64(c[b0].data_ptr(), nb, M, E, ctypes.cast(sel_h, ctypes.c_void_p),
                                             ev[b0].data_ptr(), vec[b0].data_ptr(), ws.data_ptr(), ws.numel(),
                                             N.stream_handle()),
                'acb_heevd_select_f64')
    return ev, vec


def cleansc_f64(csm: torch.Tensor, wavenumbers: torch.Tensor, steer_type: str, r_diag: bool, norm: float,
                n_iter: int = 0, damp: float = 0.6, stopn: int = 3, mpos: torch.Tensor | None = None,
                gpos: torch.Tensor | None = None, ref=None, r0: torch.Tensor | None = None,
                rm: torch.Tensor | None = None, glibc_faithful: bool = True) -> torch.Tensor:
    """CLEAN-SC for B bins: csm (B, M, M) complex128 (left unchanged: the iterations run on a copy),
    wavenumbers (B,), geometry mpos (3, M) / gpos (3, G) or given distances r0 (G,), rm (G, M)
    -> (B, G) float32, as BeamformerCleansc._calc's result rows."""
    B, M, _ = csm.shape
    if rm is None and (mpos is None or gpos is None):
        msg = 'either mpos and gpos or r0 and rm are required'
        raise ValueError(msg)
    G = int(rm.shape[0]) if rm is not None else int(gpos.shape[1])
    dev = csm.device
    p = map_params(M, G, B, steer_type, r_diag, norm, False, None if rm is not None else ref, glibc_faithful, dev)
    work = csm.to(torch.complex128).contiguous().clone()
    nbytes = N.lib().acb_cleansc_workspace_bytes(M, G, B, int(n_iter))
    if nbytes == 0:
        msg = 'invalid CLEAN-SC sizes'
        raise ValueError(msg)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    out = torch.empty((B, G), dtype=torch.float32, device=dev)
    k = wavenumbers.to(device=dev, dtype=torch.float64).contiguous()
    N.check(N.lib().acb_cleansc_f64(ctypes.byref(p), work.data_ptr(), k.data_ptr(), N.ptr(mpos), N.ptr(gpos),
                                    N.ptr(r0), N.ptr(rm), int(n_iter), float(damp), int(stopn), out.data_ptr(),
                                    ws.data_ptr(), nbytes, N.stream_handle()), 'acb_cleansc_f64')
    return out


def cleansc_custom_f64(csm: torch.Tensor, steer: torch.Tensor, r_diag: bool, norm: float, n_iter: int = 0,
                       damp: float = 0.6, stopn: int = 3) -> torch.Tensor:
    """CLEAN-SC for B bins with a steering object's own vectors: csm (B, M, M) complex128 (left unchanged),
    steer (B, G, M) complex128 (its steer_vector(f) per bin) -> (B, G) float32."""
    B, M, _ = csm.shape
    G = int(steer.shape[1])
    if steer.shape != (B, G, M) or steer.dtype != torch.complex128 or not steer.is_contiguous():
        msg = 'steer must be a contiguous complex128 (num_bins, num_grid, num_mics) tensor'
        raise ValueError(msg)
    dev = csm.device
    p = map_params(M, G, B, 'classic', r_diag, norm, False, None, False, dev)
    work = csm.to(torch.complex128).contiguous().clone()
    nbytes = N.lib().acb_cleansc_workspace_bytes(M, G, B, int(n_iter))
    if nbytes == 0:
        msg = 'invalid CLEAN-SC sizes'
        raise ValueError(msg)
    nbytes -= 16 * G * M * B          # the steering region: the vectors are given
    ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=dev)
    out = torch.empty((B, G), dtype=torch.float32, device=dev)
    N.check(N.lib().acb_cleansc_custom_f64(ctypes.byref(p), work.data_ptr(), steer.data_ptr(), int(n_iter),
                                           float(damp), int(stopn), out.data_ptr(), ws.data_ptr(), ws.numel(),
                                           N.stream_handle()), 'acb_cleansc_custom_f64')
    return out
