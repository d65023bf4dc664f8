"""Drop-ins for the reference's numba kernel entry points (acoular/fastFuncs.py), on the GPU.

* :func:`calcCSM`        -- fastFuncs.py:19-58; ``csm`` (F, M, M) c128/c64 C-contiguous is updated
  in place with ``conj(spec[f, c]) * spec[f, r]`` for r <= c; returns ``csm``.
* :func:`beamformerFreq` -- fastFuncs.py:61-214:
  ``(steerVecType, boolRemovedDiagOfCSM, normFactor, (r0, rm, k) | steer (G, M), csm | (eigval, eigvec))
  -> (map, steerNorm)`` for the predefined steering types and 'custom' steering vectors, with a full
  CSM or an eigen-decomposition tuple.
* :func:`calcPointSpreadFunction` -- fastFuncs.py:563-801; ``(steerVecType, r0, rm, k, indSource,
  dtype) -> (G, len(indSource))``.
* :func:`damasSolverGaussSeidel` -- fastFuncs.py:804-855; ``(A (..., G, G), dirtyMap (..., G), nIterations,
  relax, damasSolution (..., G))``, ``damasSolution`` overwritten with the result.

Wrong dtypes or non-contiguous arrays raise ``TypeError`` where the reference's explicit numba
signatures raise a typing error.  Every call uploads its inputs, runs the kernel and downloads the
result (these are the per-call ABI; the batched path in :mod:`acoular_b200.device` keeps data
resident).
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _native as N
from . import device as D


def _check_contig(a, dtype, name):
    if not isinstance(a, np.ndarray) or a.dtype != dtype or not a.flags.c_contiguous:
        msg = f'{name} must be a C-contiguous {np.dtype(dtype).name} array'
        raise TypeError(msg)


def calcCSM(csm: np.ndarray, SpecAllMics: np.ndarray) -> np.ndarray:  # noqa: N802, N803
    if not isinstance(csm, np.ndarray) or csm.dtype not in (np.complex128, np.complex64):
        msg = 'csm must be complex128 or complex64'
        raise TypeError(msg)
    _check_contig(csm, csm.dtype, 'csm')
    _check_contig(SpecAllMics, csm.dtype, 'SpecAllMics')
    if csm.ndim != 3 or SpecAllMics.ndim != 2 or csm.shape[0] != SpecAllMics.shape[0] or \
            csm.shape[1] != csm.shape[2] or csm.shape[1] != SpecAllMics.shape[1]:
        msg = 'csm must be (F, M, M) and SpecAllMics (F, M)'
        raise ValueError(msg)
    dev = D.require_cuda()
    c = torch.from_numpy(csm).to(dev)
    s = torch.from_numpy(SpecAllMics).to(dev)
    fn = N.lib().acb_calc_csm_c64 if csm.dtype == np.complex64 else N.lib().acb_calc_csm_c128
    N.check(fn(c.data_ptr(), s.data_ptr(), csm.shape[0], csm.shape[1], N.stream_handle()), 'calcCSM')
    csm[...] = c.cpu().numpy()
    return csm


def beamformerFreq(steerVecType, boolRemovedDiagOfCSM, normFactor, inputTupleSteer, inputTupleCsm,  # noqa: N802, N803
                   glibc_faithful: bool = True):
    if steerVecType == 'custom':
        return _beamformer_freq_custom(boolRemovedDiagOfCSM, normFactor, inputTupleSteer, inputTupleCsm)
    if steerVecType not in N.STEER_CODES:
        raise KeyError(steerVecType)
    r0, rm, k = inputTupleSteer
    if isinstance(k, np.ndarray):
        k = k.reshape(-1)[0]
    _check_contig(r0, np.float64, 'distGridToArrayCenter')
    _check_contig(rm, np.float64, 'distGridToAllMics')
    if isinstance(inputTupleCsm, tuple):
        return _beamformer_freq_eig(steerVecType, boolRemovedDiagOfCSM, normFactor, r0, rm, float(k), *inputTupleCsm,
                                    glibc_faithful=glibc_faithful)
    _check_contig(inputTupleCsm, np.complex128, 'csm')
    G, M = rm.shape
    if r0.shape != (G,) or inputTupleCsm.shape != (M, M):
        msg = 'shape mismatch between r0 (G,), rm (G, M) and csm (M, M)'
        raise ValueError(msg)
    dev = D.require_cuda()
    csm_d = torch.from_numpy(inputTupleCsm).to(dev)
    r0_d = torch.from_numpy(r0).to(dev)
    rm_d = torch.from_numpy(rm).to(dev)
    out = torch.empty(G, dtype=torch.float64, device=dev)
    nrm = torch.empty(G, dtype=torch.float64, device=dev)
    p = D.map_params(M, G, 1, steerVecType, boolRemovedDiagOfCSM, normFactor, clip_negative=False, ref=None,
                     glibc_faithful=glibc_faithful, device=dev)
    N.check(N.lib().acb_beamformer_freq_f64(ctypes.byref(p), csm_d.data_ptr(), float(k), r0_d.data_ptr(),
                                            rm_d.data_ptr(), out.data_ptr(), nrm.data_ptr(), N.stream_handle()),
            'beamformerFreq')
    return out.cpu().numpy(), nrm.cpu().numpy()


def _beamformer_freq_eig(steer_type, r_diag, norm, r0, rm, k, eigval, eigvec, glibc_faithful=True):
    """beamformerFreq with an eigen tuple (eigVal[E] float64, eigVec[M, E] complex128):
    _freqBeamformer_EigValues (acoular/fastFuncs.py:313-411) on the device."""
    eigval = np.asarray(eigval)
    eigvec = np.ascontiguousarray(eigvec)
    _check_contig(eigval, np.float64, 'eigVal')
    if eigvec.dtype != np.complex128:
        msg = 'eigVec must be complex128'
        raise TypeError(msg)
    G, M = rm.shape
    E = eigval.shape[0]
    if r0.shape != (G,) or eigvec.shape != (M, E):
        msg = 'shape mismatch between r0 (G,), rm (G, M), eigVal (E,) and eigVec (M, E)'
        raise ValueError(msg)
    dev = D.require_cuda()
    ev_d = torch.from_numpy(eigval).to(dev)
    evec_d = torch.from_numpy(eigvec).to(dev)
    r0_d = torch.from_numpy(r0).to(dev)
    rm_d = torch.from_numpy(rm).to(dev)
    out = torch.empty(G, dtype=torch.float64, device=dev)
    nrm = torch.empty(G, dtype=torch.float64, device=dev)
    p = D.map_params(M, G, 1, steer_type, r_diag, norm, clip_negative=False, ref=None, glibc_faithful=glibc_faithful,
                     device=dev)
    N.check(N.lib().acb_beamformer_freq_eig_f64(ctypes.byref(p), E, ev_d.data_ptr(), evec_d.data_ptr(), float(k),
                                                r0_d.data_ptr(), rm_d.data_ptr(), out.data_ptr(), nrm.data_ptr(),
                                                N.stream_handle()), 'beamformerFreq')
    return out.cpu().numpy(), nrm.cpu().numpy()


def _beamformer_freq_custom(r_diag, norm, steer_vec, csm_or_eig):
    """beamformerFreq('custom', ...) with a (G, M) complex128 steering matrix (acoular/fastFuncs.py:414-559)."""
    h = np.asarray(steer_vec)
    if h.dtype != np.complex128 or h.ndim != 2:
        msg = 'custom steering vectors must be a (num_grid, num_mics) complex128 array'
        raise TypeError(msg)
    G, M = h.shape
    dev = D.require_cuda()
    h_d = torch.from_numpy(np.ascontiguousarray(h)).to(dev)[None]
    out = torch.empty((1, G), dtype=torch.float64, device=dev)
    nrm = torch.empty((1, G), dtype=torch.float64, device=dev)
    if isinstance(csm_or_eig, tuple):
        ev, evec = csm_or_eig
        ev = np.ascontiguousarray(ev, dtype=np.float64)
        evec = np.ascontiguousarray(evec, dtype=np.complex128)
        if evec.shape != (M, ev.shape[0]):
            msg = 'eigVec must be (num_mics, num_eigs)'
            raise ValueError(msg)
        eig = (torch.from_numpy(ev).to(dev)[None], torch.from_numpy(evec).to(dev)[None])
        D.map_custom_f64(None, h_d, r_diag, float(norm), out=out, steer_norm=nrm, eig=eig)
    else:
        _check_contig(csm_or_eig, np.complex128, 'csm')
        if csm_or_eig.shape != (M, M):
            msg = 'csm must be (num_mics, num_mics)'
            raise ValueError(msg)
        c = torch.from_numpy(csm_or_eig).to(dev)[None]
        D.map_custom_f64(c, h_d, r_diag, float(norm), out=out, steer_norm=nrm)
    return out[0].cpu().numpy(), nrm[0].cpu().numpy()


def calcPointSpreadFunction(steerVecType, distGridToArrayCenter, distGridToAllMics, waveNumber, indSource,  # noqa: N802, N803
                            dtype):
    """PSF of unit sources at the grid points ``indSource``: (G, len(indSource)) of ``dtype``."""
    if steerVecType not in N.STEER_CODES or steerVecType == 'custom':
        raise KeyError(steerVecType)
    dev = D.require_cuda()
    rm = torch.as_tensor(np.ascontiguousarray(np.atleast_2d(distGridToAllMics), dtype=np.float64), device=dev)
    r0 = torch.as_tensor(np.array(np.broadcast_to(distGridToArrayCenter, (rm.shape[0],)), dtype=np.float64),
                         device=dev)
    k = float(np.asarray(waveNumber).reshape(-1)[0])
    src = np.asarray(indSource, dtype=np.int64).reshape(-1)
    out = D.psf_f64(r0, rm, k, src, steerVecType, round_f32=np.dtype(dtype) == np.float32)
    return out.cpu().numpy().astype(dtype)


def damasSolverGaussSeidel(A, dirtyMap, nIterations, relax, damasSolution):  # noqa: N802, N803
    """Gauss-Seidel DAMAS solver; ``damasSolution`` (float64, C-contiguous) holds the start and is
    overwritten with the result after ``nIterations`` sweeps."""
    _check_contig(damasSolution, np.float64, 'damasSolution')
    dev = D.require_cuda()
    y = np.asarray(dirtyMap, dtype=np.float64)
    G = y.shape[-1]
    B = int(np.prod(y.shape[:-1], dtype=np.int64))
    if damasSolution.shape != y.shape or np.shape(A) != y.shape + (G,):
        msg = 'A must be (..., G, G) and dirtyMap / damasSolution (..., G)'
        raise ValueError(msg)
    A_d = torch.as_tensor(np.ascontiguousarray(A, dtype=np.float64).reshape(B, G, G), device=dev)
    y_d = torch.as_tensor(np.ascontiguousarray(y).reshape(B, G), device=dev)
    x_d = torch.as_tensor(damasSolution.reshape(B, G), device=dev).clone()
    D.damas_gauss_seidel(A_d, y_d, int(np.asarray(nIterations).reshape(-1)[0]),
                         float(np.asarray(relax).reshape(-1)[0]), x_d)
    damasSolution[...] = x_d.cpu().numpy().reshape(damasSolution.shape)
    return damasSolution
