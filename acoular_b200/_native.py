"""ctypes binding of the C ABI in ``include/acoular_b200.h`` (``lib/libacoular_b200.so``).

The library is required: importing the device path without it raises ``ImportError``; there is no
CPU fallback.  Device buffers are torch CUDA tensors; their ``data_ptr()`` and the current torch
stream handle are what crosses the boundary.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / 'lib' / 'libacoular_b200.so'

ACB_OK = 0
ACB_ERR_SHAPE, ACB_ERR_ARG, ACB_ERR_CUDA, ACB_ERR_UNSUPPORTED, ACB_ERR_WORKSPACE, ACB_ERR_TIMEOUT = 1, 2, 3, 4, 5, 6
STATUS_NAMES = {0: 'ok', 1: 'ACB_ERR_SHAPE', 2: 'ACB_ERR_ARG', 3: 'ACB_ERR_CUDA', 4: 'ACB_ERR_UNSUPPORTED',
                5: 'ACB_ERR_WORKSPACE', 6: 'ACB_ERR_TIMEOUT'}
STEER_CODES = {'classic': 1, 'inverse': 2, 'true level': 3, 'true location': 4}
C128, C64 = 0, 1
CSM_TC_TF32, CSM_TC_BF16X3 = 2, 3     # tensor-core CSM forms (complex128 csm_upper)
TC_PRECISIONS = {'bf16x3': 0, 'tf32': 1, 'fp16': 2}
F32, F64 = 0, 1


class AcbError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        text = lib().acb_status_string(status).decode()
        extra = ''
        if status == 3:
            extra = ': ' + lib().acb_last_cuda_error().decode()
        super().__init__(f'{where}: {STATUS_NAMES.get(status, status)} ({text}{extra})')


class MapParams(ctypes.Structure):
    _fields_ = [
        ('num_mics', ctypes.c_int),
        ('num_grid', ctypes.c_int64),
        ('num_bins', ctypes.c_int),
        ('steer_type', ctypes.c_int),
        ('r_diag', ctypes.c_int),
        ('clip_negative', ctypes.c_int),
        ('norm', ctypes.c_double),
        ('ref_mode', ctypes.c_int),
        ('ref_point', ctypes.c_double * 3),
        ('ref_distance', ctypes.c_double),
        ('glibc_faithful', ctypes.c_int),
        ('sincos_table', ctypes.c_void_p),
        ('sincos_table_slots', ctypes.c_int64),
        ('tc_pass_chunks', ctypes.c_int),
        ('tc_splits', ctypes.c_int),
    ]


class MapIO(ctypes.Structure):
    _fields_ = [
        ('csm', ctypes.c_void_p),
        ('wavenumber', ctypes.c_void_p),
        ('mpos', ctypes.c_void_p),
        ('gpos', ctypes.c_void_p),
        ('out_map', ctypes.c_void_p),
        ('out_steer_norm', ctypes.c_void_p),
    ]


_lib = None

_VP = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_D = ctypes.c_double
_SZ = ctypes.c_size_t

# name -> (restype, argtypes): every symbol declared in include/acoular_b200.h
SIGNATURES = {
    'acb_status_string': (ctypes.c_char_p, [_I]),
    'acb_abi_version': (_I, []),
    'acb_last_cuda_error': (ctypes.c_char_p, []),
    'acb_calc_csm_c128': (_I, [_VP, _VP, _I, _I, _VP]),
    'acb_calc_csm_c64': (_I, [_VP, _VP, _I, _I, _VP]),
    'acb_csm_workspace_bytes': (_SZ, [_I, _I, _I64, _I]),
    'acb_csm_workspace_bytes_block': (_SZ, [_I, _I, _I64, _I, _I]),
    'acb_csm_accumulate': (_I, [_VP, _I, _I64, _I, _I, _I, _I64, _I64, _VP, _VP, _I, _I, _I, _VP, _VP, _SZ, _VP]),
    'acb_csm_finalize': (_I, [_VP, _I, _I, _I, _D, _VP, _VP]),
    'acb_map_f64': (_I, [ctypes.POINTER(MapParams), _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    'acb_beamformer_freq_f64': (_I, [ctypes.POINTER(MapParams), _VP, _D, _VP, _VP, _VP, _VP, _VP]),
    'acb_map_eig_f64': (_I, [ctypes.POINTER(MapParams), _I, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    'acb_map_rm_f64': (_I, [ctypes.POINTER(MapParams), _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    'acb_spectra_workspace_bytes': (ctypes.c_size_t, [_I, _I, ctypes.c_int64]),
    'acb_spectra': (_I, [_VP, _I, ctypes.c_int64, _I, _I, _I, ctypes.c_int64, ctypes.c_int64, _VP, _VP, _I, _D, _I,
                         _VP, _VP, ctypes.c_size_t, _VP]),
    'acb_auto_spectra': (_I, [_VP, ctypes.c_int64, _I, _I, _D, _VP, _VP]),
    'acb_cross_spectra': (_I, [_VP, ctypes.c_int64, _I, _I, _I, _D, _VP, _VP]),
    'acb_cleansc_workspace_bytes': (ctypes.c_size_t, [_I, ctypes.c_int64, _I, _I]),
    'acb_heevd_workspace_bytes': (ctypes.c_size_t, [_I, _I]),
    'acb_heevd_f64': (_I, [_VP, _I, _I, _VP, _VP, _VP, _VP, ctypes.c_size_t, _VP]),
    'acb_heevd_select_f64': (_I, [_VP, _I, _I, _I, _VP, _VP, _VP, _VP, ctypes.c_size_t, _VP]),
    'acb_cleansc_f64': (_I, [ctypes.POINTER(MapParams), _VP, _VP, _VP, _VP, _VP, _VP, _I, _D, _I, _VP, _VP,
                             ctypes.c_size_t, _VP]),
    'acb_cleansc_custom_f64': (_I, [ctypes.POINTER(MapParams), _VP, _VP, _I, _D, _I, _VP, _VP, ctypes.c_size_t,
                                    _VP]),
    'acb_psf_f64': (_I, [ctypes.POINTER(MapParams), _I, _VP, _D, _VP, _VP, _I, _VP, _VP]),
    'acb_damas_gauss_seidel_f64': (_I, [_VP, ctypes.c_int64, _I, _VP, _VP, _I, _D, _I, _VP]),
    'acb_map_custom_f64': (_I, [ctypes.POINTER(MapParams), _VP, _VP, _VP, _VP, _VP]),
    'acb_map_eig_custom_f64': (_I, [ctypes.POINTER(MapParams), _I, _VP, _VP, _VP, _VP, _VP, _VP]),
    'acb_beamformer_freq_eig_f64': (_I, [ctypes.POINTER(MapParams), _I, _VP, _VP, _D, _VP, _VP, _VP, _VP, _VP]),
    'acb_sincos_table_build_host': (_I64, [_VP, _I64, ctypes.c_float, _I]),
    'acb_map_tc_workspace_bytes': (_SZ, [_I, _I, _I]),
    'acb_tc_set_wait_limit_ns': (ctypes.c_uint64, [ctypes.c_uint64]),
    'acb_map_tc': (_I, [ctypes.POINTER(MapParams), _I, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _SZ, _VP, _VP]),
    'acb_map_tc_noalloc': (_I, [ctypes.POINTER(MapParams), _I, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    'acb_map_tc_batch_workspace_bytes': (_SZ, [ctypes.POINTER(MapParams), _I, _I]),
    'acb_map_tc_batch': (_I, [ctypes.POINTER(MapParams), ctypes.POINTER(MapIO), _I, _I, _VP, _SZ, _VP, _VP]),
}


def lib():
    """Load the native library (raises ``ImportError`` if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            msg = (f'acoular_b200 native library missing at {LIB_PATH}; build it with '
                   '`python -m acoular_b200.build` (nvcc, sm_100a)')
            raise ImportError(msg)
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, where: str) -> None:
    if status != ACB_OK:
        raise AcbError(status, where)


def ptr(t) -> int | None:
    """Device pointer of a torch tensor (None for None)."""
    if t is None:
        return None
    return t.data_ptr()


def stream_handle(stream=None) -> int | None:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def exported_symbols() -> list[str]:
    return list(SIGNATURES)


def header_symbols() -> list[str]:
    """Function names declared in include/acoular_b200.h (parsed from the header text)."""
    import re
    hdr = (_PKG.parent / 'include' / 'acoular_b200.h').read_text()
    hdr = re.sub(r'/\*.*?\*/', '', hdr, flags=re.S)
    return sorted(set(re.findall(r'\b(acb_[a-z0-9_]+)\s*\(', hdr)))


def nproc() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1
