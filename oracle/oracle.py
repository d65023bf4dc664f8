"""CPU oracle for the Acoular frequency-domain beamforming path.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py``, always as the checker or the timed CPU reference -- never by the product
package ``acoular_b200``.

This module restates the reference's (Acoular 26.08) host-side glue for the path in numpy and
calls the C restatement of its numba kernels in ``oracle_core.c`` (built into
``oracle/lib/liboracle_acoular.so`` by ``oracle/build_oracle.sh``):

* :func:`source_windows`   -- ``BaseSpectra._get_source_data``   acoular/spectra.py:171-184
* :func:`num_blocks`       -- ``PowerSpectra._get_num_blocks``   acoular/spectra.py:281-283
* :func:`fftfreq`          -- ``BaseSpectra.fftfreq``            acoular/spectra.py:128-168
* :func:`calc_csm`         -- ``PowerSpectra.calc_csm``          acoular/spectra.py:366-416
* :func:`dist_mat`         -- ``dist_mat``                       acoular/environments.py:65-103
* :func:`beamformer_freq`  -- ``beamformerFreq`` (full CSM)      acoular/fastFuncs.py:61-214, 217-311
* :func:`sig_loss_norm`    -- ``BeamformerBase.sig_loss_norm``   acoular/fbeamform.py:438-451
* :func:`beamformer_calc`  -- ``BeamformerBase._calc``           acoular/fbeamform.py:475-510
* :func:`synthetic`        -- ``BeamformerBase.synthetic``       acoular/fbeamform.py:512-593
* :func:`L_p`              -- ``L_p``                            acoular/fbeamform.py:2412-2429

Parity of the oracle itself is pinned by ``tests/test_oracle.py`` against goldens generated by
running the reference's own code (``tests/golden/make_golden.py``).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np
from scipy import fft as sfft

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / 'lib' / 'liboracle_acoular.so'
_lib = None

WINDOWS = {
    'Rectangular': np.ones,
    'Hanning': np.hanning,
    'Hamming': np.hamming,
    'Bartlett': np.bartlett,
    'Blackman': np.blackman,
}
OVERLAPS = {'None': 1, '50%': 2, '75%': 4, '87.5%': 8}
STEER_TYPES = {'classic': 1, 'inverse': 2, 'true level': 3, 'true location': 4}


def build(force: bool = False) -> Path:
    """Compile ``oracle_core.c`` with gcc (no GPU needed)."""
    if force or not _LIB_PATH.exists() or _LIB_PATH.stat().st_mtime < (_HERE / 'oracle_core.c').stat().st_mtime:
        subprocess.run(['bash', str(_HERE / 'build_oracle.sh')], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(_LIB_PATH))
        dp = ctypes.POINTER(ctypes.c_double)
        fp = ctypes.POINTER(ctypes.c_float)
        i64 = ctypes.c_int64
        L.orc_calc_csm_c128.argtypes = [dp, dp, i64, i64]
        L.orc_calc_csm_c64.argtypes = [fp, fp, i64, i64]
        L.orc_calc_csm_blocks_c128.argtypes = [dp, dp, i64, i64, i64]
        L.orc_calc_csm_blocks_c64.argtypes = [fp, fp, i64, i64, i64]
        L.orc_dist_mat.argtypes = [dp, dp, i64, i64, dp]
        L.orc_beamformer_fullcsm.argtypes = [dp, dp, dp, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                             ctypes.c_int, i64, i64, dp, dp]
        L.orc_beamformer_eig.argtypes = [dp, dp, dp, dp, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                         i64, i64, i64, dp, dp]
        L.orc_beamformer_custom.argtypes = [dp, dp, dp, i64, dp, ctypes.c_double, ctypes.c_int, i64, i64, dp, dp]
        L.orc_psf.argtypes = [dp, dp, ctypes.c_double, ctypes.POINTER(i64), i64, ctypes.c_int, i64, i64, dp]
        L.orc_damas_gauss_seidel_bins.argtypes = [dp, dp, i64, i64, i64, ctypes.c_double, dp]
        L.orc_transfer.argtypes = [dp, dp, ctypes.c_double, i64, i64, dp]
        L.orc_num_threads.restype = ctypes.c_int
        L.orc_set_num_threads.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def num_threads() -> int:
    return lib().orc_num_threads()


def set_num_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


# ----------------------------------------------------------------------------------------------
# Stage A: cross-spectral matrix
# ----------------------------------------------------------------------------------------------
def _source_blocks(samples: np.ndarray, num: int):
    """``TimeSamples.result(num)`` (acoular/sources.py:417-467): consecutive blocks, last one short."""
    n = samples.shape[0]
    i = 0
    while i < n:
        yield samples[i:i + num]
        i += num


def source_windows(samples: np.ndarray, block_size: int, overlap: int):
    """Overlapped windows as yielded by ``_get_source_data`` (acoular/spectra.py:171-184)."""
    bs = block_size
    temp = np.empty((2 * bs, samples.shape[1]))
    pos = bs
    posinc = bs / overlap
    for data_block in _source_blocks(samples, bs):
        ns = data_block.shape[0]
        temp[bs:bs + ns] = data_block
        while pos + bs <= bs + ns:
            yield temp[int(pos):int(pos + bs)]
            pos += posinc
        temp[0:bs] = temp[bs:]
        pos -= bs


def num_blocks(num_samples: int, block_size: int, overlap: int) -> float:
    """acoular/spectra.py:281-283 -- a float formula, not a count."""
    return overlap * num_samples / block_size - overlap + 1


def fftfreq(block_size: int, sample_freq: float) -> np.ndarray:
    """acoular/spectra.py:128-168."""
    return abs(sfft.fftfreq(block_size, 1.0 / sample_freq)[: int(block_size / 2 + 1)])


def calc_csm(samples: np.ndarray, block_size: int = 1024, window: str = 'Rectangular', overlap: str = 'None',
             precision: str = 'complex128', return_spectra: bool = False):
    """``PowerSpectra.calc_csm`` (acoular/spectra.py:366-416) with the C ``calcCSM``."""
    ov = OVERLAPS[overlap]
    wind = WINDOWS[window](block_size)
    weight = np.dot(wind, wind)
    wind = wind[np.newaxis, :].swapaxes(0, 1)
    numfreq = int(block_size / 2 + 1)
    M = samples.shape[1]
    csm_upper = np.zeros((numfreq, M, M), dtype=precision)
    L = lib()
    spectra = []
    for data in source_windows(samples, block_size, ov):
        ft = np.ascontiguousarray(sfft.rfft(data * wind, None, 0).astype(precision))
        if return_spectra:
            spectra.append(ft.copy())
        if precision == 'complex128':
            L.orc_calc_csm_c128(_dp(csm_upper), _dp(ft), numfreq, M)
        else:
            L.orc_calc_csm_c64(_fp(csm_upper), _fp(ft), numfreq, M)
    csm_lower = csm_upper.conj().transpose(0, 2, 1)
    for f in range(csm_lower.shape[0]):
        np.fill_diagonal(csm_lower[f], 0)
    csm = csm_lower + csm_upper
    out = csm * (2.0 / block_size / weight / num_blocks(samples.shape[0], block_size, ov))
    if return_spectra:
        return out, spectra
    return out


# ----------------------------------------------------------------------------------------------
# Geometry
# ----------------------------------------------------------------------------------------------
def dist_mat(gpos: np.ndarray, mpos: np.ndarray) -> np.ndarray:
    """acoular/environments.py:65-103; gpos (3, N), mpos (3, M) -> (N, M)."""
    gpos = np.ascontiguousarray(gpos, dtype=np.float64)
    mpos = np.ascontiguousarray(mpos, dtype=np.float64)
    N, M = gpos.shape[1], mpos.shape[1]
    rm = np.empty((N, M))
    lib().orc_dist_mat(_dp(gpos), _dp(mpos), N, M, _dp(rm))
    return rm


def apparent_r(gpos, mpos=0.0):
    """``Environment.apparent_r`` (acoular/environments.py:202-238)."""
    if np.isscalar(mpos):
        mpos = np.array((0, 0, 0), dtype=np.float64)[:, np.newaxis]
    rm = dist_mat(gpos, mpos)
    if rm.shape[1] == 1:
        rm = rm[:, 0]
    return rm


def rect_grid_pos(x_min, x_max, y_min, y_max, z, increment):
    """``RectGrid`` nxsteps/nysteps/pos (acoular/grids.py:332-358)."""
    i = abs(increment)
    nx = round((abs(x_max - x_min) + i) / i) if i != 0 else 1
    ny = round((abs(y_max - y_min) + i) / i) if i != 0 else 1
    bpos = np.mgrid[x_min:x_max:nx * 1j, y_min:y_max:ny * 1j, z:z + 0.1]
    bpos.resize((3, nx * ny))
    return bpos, (nx, ny)


def rect_grid3d_pos(x_min, x_max, y_min, y_max, z_min, z_max, increment):
    """``RectGrid3D`` (acoular/grids.py:523-560), scalar increment."""
    i = abs(increment)
    nx = round((abs(x_max - x_min) + i) / i)
    ny = round((abs(y_max - y_min) + i) / i)
    nz = round((abs(z_max - z_min) + i) / i)
    bpos = np.mgrid[x_min:x_max:nx * 1j, y_min:y_max:ny * 1j, z_min:z_max:nz * 1j]
    bpos.resize((3, nx * ny * nz))
    return bpos, (nx, ny, nz)


# ----------------------------------------------------------------------------------------------
# Stage B: steered-response map
# ----------------------------------------------------------------------------------------------
def beamformer_freq(steer_type: str, r_diag: bool, norm: float, r0: np.ndarray, rm: np.ndarray, k: float,
                    csm: np.ndarray):
    """``beamformerFreq`` for the predefined steering types and a full CSM (fastFuncs.py:61-214)."""
    csm = np.ascontiguousarray(csm, dtype=np.complex128)
    r0 = np.ascontiguousarray(r0, dtype=np.float64)
    rm = np.ascontiguousarray(rm, dtype=np.float64)
    G, M = rm.shape
    res = np.zeros(G)
    nrm = np.zeros(G)
    lib().orc_beamformer_fullcsm(_dp(csm), _dp(r0), _dp(rm), float(k), float(norm), int(bool(r_diag)),
                                 STEER_TYPES[steer_type], G, M, _dp(res), _dp(nrm))
    return res, nrm


def beamformer_freq_eig(steer_type: str, r_diag: bool, norm: float, r0: np.ndarray, rm: np.ndarray, k: float,
                        eigval: np.ndarray, eigvec: np.ndarray):
    """``beamformerFreq`` with an eigen-decomposition tuple ``(eigval[E], eigvec[M, E])``
    (fastFuncs.py:61-214 dispatching to _freqBeamformer_EigValues, fastFuncs.py:313-411)."""
    eigval = np.ascontiguousarray(eigval, dtype=np.float64)
    eigvec = np.ascontiguousarray(eigvec, dtype=np.complex128)
    r0 = np.ascontiguousarray(r0, dtype=np.float64)
    rm = np.ascontiguousarray(rm, dtype=np.float64)
    G, M = rm.shape
    E = eigval.shape[0]
    res = np.zeros(G)
    nrm = np.zeros(G)
    lib().orc_beamformer_eig(_dp(eigval), _dp(eigvec), _dp(r0), _dp(rm), float(k), float(norm), int(bool(r_diag)),
                             STEER_TYPES[steer_type], G, M, E, _dp(res), _dp(nrm))
    return res, nrm


def beamformer_freq_custom(r_diag: bool, norm: float, steer: np.ndarray, csm=None, eig=None):
    """``beamformerFreq('custom', ...)`` (fastFuncs.py:414-559): steer (G, M) complex128 with a full CSM
    (M, M) or an eigen tuple (eigval[E], eigvec[M, E])."""
    steer = np.ascontiguousarray(steer, dtype=np.complex128)
    G, M = steer.shape
    res = np.zeros(G)
    nrm = np.zeros(G)
    if eig is None:
        c = np.ascontiguousarray(csm, dtype=np.complex128)
        lib().orc_beamformer_custom(_dp(c), None, None, 0, _dp(steer), float(norm), int(bool(r_diag)), G, M,
                                    _dp(res), _dp(nrm))
    else:
        ev = np.ascontiguousarray(eig[0], dtype=np.float64)
        evec = np.ascontiguousarray(eig[1], dtype=np.complex128)
        lib().orc_beamformer_custom(None, _dp(ev), _dp(evec), ev.shape[0], _dp(steer), float(norm),
                                    int(bool(r_diag)), G, M, _dp(res), _dp(nrm))
    return res, nrm


def uniform_flow_apparent_r(gpos, mpos, ma: float, fdv):
    """``UniformFlowEnvironment.apparent_r`` (acoular/environments.py:290-332): path length r and its
    angle theta to the flow direction give r / (sqrt(ma^2 cos^2 theta - ma^2 + 1) - ma cos theta)."""
    if np.isscalar(mpos):
        mpos = np.array((0, 0, 0), dtype=np.float32)[:, np.newaxis]
    fdv = np.asarray(fdv, dtype=np.float64)
    u = fdv / np.sqrt((fdv * fdv).sum())
    d = np.asarray(gpos)[:, :, np.newaxis] - np.asarray(mpos)[:, np.newaxis, :]
    r = np.sqrt(np.sum(d * d, 0))
    mc = (ma * np.sum(d.reshape((3, -1)) * u[:, np.newaxis], 0) / r.reshape(-1)).reshape(r.shape)
    r = r * (1 / (-mc + np.sqrt(mc * mc - ma * ma + 1)))
    if r.shape[1] == 1:
        r = r[:, 0]
    return r


def eig_na(n: int, num_mics: int) -> int:
    """``BeamformerEig.na`` (acoular/fbeamform.py:844-850)."""
    na = n
    if na < 0:
        na = max(num_mics + na, 0)
    return min(num_mics - 1, na)


def beamformer_eig_calc(eigvals, eigvecs, freqs, ind, r0, rm, c: float, steer_type: str, r_diag: bool, n: int = -1,
                        r_diag_norm: float = 0.0, out=None):
    """``BeamformerEig._calc`` (acoular/fbeamform.py:852-888): component ``na`` of each bin's eigh."""
    G, M = rm.shape
    if out is None:
        out = np.zeros((eigvals.shape[0], G))
    na = eig_na(n, M)
    norm = sig_loss_norm(r_diag, M, r_diag_norm)
    for i in ind:
        b = beamformer_freq_eig(steer_type, r_diag, norm, r0, rm, 2 * np.pi * freqs[i] / c,
                                np.array(eigvals[i], dtype='float64')[na:na + 1],
                                np.array(eigvecs[i], dtype='complex128')[:, na:na + 1])[0]
        if r_diag:
            b[np.sign(b) < 0] = 0.0
        out[i] = b
    return out


def beamformer_music_calc(eigvals, eigvecs, freqs, ind, r0, rm, c: float, steer_type: str, n: int = 1, out=None):
    """``BeamformerMusic._calc`` (acoular/fbeamform.py:911-944): the M - na smallest components,
    full CSM, normalised to 4e-10 * min / map."""
    G, M = rm.shape
    if out is None:
        out = np.zeros((eigvals.shape[0], G))
    ne = int(M - eig_na(n, M))
    norm = sig_loss_norm(False, M, 1.0) * M ** 2
    for i in ind:
        b = beamformer_freq_eig(steer_type, False, norm, r0, rm, 2 * np.pi * freqs[i] / c,
                                np.array(eigvals[i], dtype='float64')[:ne],
                                np.array(eigvecs[i], dtype='complex128')[:, :ne])[0]
        out[i] = 4e-10 * b.min() / b
    return out


def psf(steer_type: str, r0: np.ndarray, rm: np.ndarray, k: float, ind, precision: str = 'float64'):
    """``calcPointSpreadFunction`` (fastFuncs.py:563-801): (G, len(ind)) PSF of unit sources at the grid
    points ``ind``, cast to ``precision`` as its output array is."""
    r0 = np.ascontiguousarray(r0, dtype=np.float64)
    rm = np.ascontiguousarray(rm, dtype=np.float64)
    src = np.ascontiguousarray(ind, dtype=np.int64)
    G, M = rm.shape
    out = np.zeros((G, src.shape[0]))
    lib().orc_psf(_dp(r0), _dp(rm), float(k), src.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), src.shape[0],
                  STEER_TYPES[steer_type], G, M, _dp(out))
    return out.astype(precision)


def damas_gauss_seidel(A: np.ndarray, y: np.ndarray, n_iter: int, relax: float, x: np.ndarray) -> np.ndarray:
    """``damasSolverGaussSeidel`` (fastFuncs.py:804-855) over leading bin axes: A (..., G, G),
    y and x (..., G); x is the starting solution and is overwritten with the result (returned)."""
    A = np.ascontiguousarray(A, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    G = y.shape[-1]
    F = int(np.prod(y.shape[:-1], dtype=np.int64))
    xs = np.ascontiguousarray(x, dtype=np.float64).copy()
    lib().orc_damas_gauss_seidel_bins(_dp(A), _dp(y), F, G, int(n_iter), float(relax), _dp(xs))
    x[...] = xs
    return x


def beamformer_damas_calc(csm, freqs, ind, r0, rm, c: float, steer_type: str, r_diag: bool, n_iter: int = 100,
                          damp: float = 1.0, psf_precision: str = 'float64', r_diag_norm: float = 0.0, out=None):
    """``BeamformerDamas._calc`` (acoular/fbeamform.py:1167-1208) for a plain ``SteeringVector``: the
    conventional map (negative values set to 0 with r_diag) deconvolved by Gauss-Seidel with the full PSF."""
    G, M = rm.shape
    if out is None:
        out = np.zeros((csm.shape[0], G))
    normfactor = sig_loss_norm(r_diag, M, r_diag_norm)
    for i in ind:
        k = 2 * np.pi * freqs[i] / c
        y = beamformer_freq(steer_type, r_diag, normfactor, r0, rm, k, np.array(csm[i], dtype='complex128'))[0]
        if r_diag:
            y[np.sign(y) < 0] = 0.0
        x = y.copy()
        A = psf(steer_type, r0, rm, k, np.arange(G), psf_precision)
        out[i] = damas_gauss_seidel(A, y, n_iter, damp, x)
    return out


def transfer(r0, rm, k: float) -> np.ndarray:
    """``calcTransfer`` (fastFuncs.py:857-897): (G, M) complex128 transfer functions."""
    rm = np.ascontiguousarray(np.atleast_2d(rm), dtype=np.float64)
    r0 = np.ascontiguousarray(np.broadcast_to(r0, (rm.shape[0],)), dtype=np.float64)
    out = np.zeros(rm.shape, dtype=np.complex128)
    lib().orc_transfer(_dp(r0), _dp(rm), float(k), rm.shape[0], rm.shape[1], _dp(out))
    return out


STEER_FUNCS = {   # SteeringVector._steer_funcs_freq (acoular/fbeamform.py:145-153)
    'classic': lambda x: x / np.abs(x) / x.shape[-1],
    'inverse': lambda x: 1.0 / x.conj() / x.shape[-1],
    'true level': lambda x: x / np.einsum('ij,ij->i', x, x.conj())[:, np.newaxis],
    'true location': lambda x: x / np.sqrt(np.einsum('ij,ij->i', x, x.conj()) * x.shape[-1])[:, np.newaxis],
}


def steer_vector(steer_type: str, r0, rm, k: float, ind=None) -> np.ndarray:
    """``SteeringVector.steer_vector`` (fbeamform.py:233-258) through ``transfer`` (207-231)."""
    if ind is not None:
        r0, rm = np.atleast_1d(np.asarray(r0)[ind]), np.atleast_2d(np.asarray(rm)[ind])
    return STEER_FUNCS[steer_type](transfer(r0, rm, k))


def beamformer_functional_calc(eigvals, eigvecs, freqs, ind, r0, rm, c: float, steer_type: str, gamma: float,
                               out=None):
    """``BeamformerFunctional._calc`` (acoular/fbeamform.py:712-786), full CSM: eigenvalues to the power
    1/gamma, the eigen map divided by the steering norm, to the power gamma, times the norm."""
    G, M = rm.shape
    if out is None:
        out = np.zeros((eigvals.shape[0], G))
    normfactor = sig_loss_norm(False, M, 1.0)
    for i in ind:
        with np.errstate(invalid='ignore'):
            ev = np.array(eigvals[i], dtype='float64') ** (1.0 / gamma)
        bo, sn = beamformer_freq_eig(steer_type, False, 1.0, r0, rm, 2 * np.pi * freqs[i] / c, ev,
                                     np.array(eigvecs[i], dtype='complex128'))
        bo /= sn
        with np.errstate(invalid='ignore'):
            out[i] = (bo ** gamma) * sn * normfactor
    return out


def beamformer_orth_calc(eigvals, eigvecs, freqs, ind, r0, rm, c: float, steer_type: str, r_diag: bool, eva_list,
                         r_diag_norm: float = 0.0, out=None):
    """``BeamformerOrth._calc`` (acoular/fbeamform.py:1366-1388): for each listed eigen-component, its
    eigenvalue / num_mics is added at the argmax of that component's map."""
    G, M = rm.shape
    if out is None:
        out = np.zeros((eigvals.shape[0], G))
    normfactor = sig_loss_norm(r_diag, M, r_diag_norm)
    for i in ind:
        ev = np.array(eigvals[i], dtype='float64')
        evec = np.array(eigvecs[i], dtype='complex128')
        for n in eva_list:
            bo = beamformer_freq_eig(steer_type, r_diag, normfactor, r0, rm, 2 * np.pi * freqs[i] / c, np.ones(1),
                                     np.ascontiguousarray(evec[:, n].reshape((-1, 1))))[0]
            out[i, bo.argmax()] += ev[n] / M
    return out


def beamformer_cleansc_calc(csm, freqs, ind, r0, rm, c: float, steer_type: str, r_diag: bool, n_iter: int = 0,
                            damp: float = 0.6, stopn: int = 3, r_diag_norm: float = 0.0, out=None):
    """``BeamformerCleansc._calc`` (acoular/fbeamform.py:1424-1490): per bin, CLEAN-SC iterations on the
    conventional map; the result (float32, like the reference's) holds damp * peak at each peak."""
    G, M = rm.shape
    if out is None:
        out = np.zeros((csm.shape[0], G))
    normfactor = sig_loss_norm(r_diag, M, r_diag_norm)
    result = np.zeros(G, 'f')
    J = M * 2 if not n_iter else n_iter
    powers = np.zeros(J, 'd')
    for i in ind:
        k = 2 * np.pi * freqs[i] / c
        cs = np.array(csm[i], dtype='complex128', copy=True)
        h = beamformer_freq(steer_type, r_diag, normfactor, r0, rm, k, cs)[0]
        result *= 0.0
        for j in range(J):
            xi_max = h.argmax()
            powers[j] = hmax = h[xi_max]
            result[xi_max] += damp * hmax
            if j > stopn and hmax > powers[j - stopn]:
                break
            wmax = steer_vector(steer_type, r0, rm, k, xi_max) * np.sqrt(normfactor)
            wmax = wmax[0].conj()
            hh = wmax.copy()
            D1 = np.dot(cs.T - np.diag(np.diag(cs)), wmax) / hmax
            ww = wmax.conj() * wmax
            for _ in range(20):
                H = hh.conj() * hh
                hh = (D1 + H * wmax) / np.sqrt(1 + np.dot(ww, H))
            hh = hh[:, np.newaxis]
            csm1 = hmax * (hh * hh.conj().T)
            h1 = beamformer_freq_eig(steer_type, r_diag, normfactor, r0, rm, k, np.array((hmax,)),
                                     np.ascontiguousarray(hh.conj()))[0]
            h -= damp * h1
            cs -= damp * csm1.T
        out[i] = result
    return out


def beamformer_cleansc_custom_calc(csm, freqs, ind, steer_vectors, r_diag: bool, n_iter: int = 0, damp: float = 0.6,
                                   stopn: int = 3, r_diag_norm: float = 0.0, out=None):
    """``BeamformerCleansc._calc`` (acoular/fbeamform.py:1424-1490) with a steering object of its own
    (``_beamformer_params`` routes it as 'custom', acoular/fbeamform.py:470-472): ``steer_vectors(f)`` gives
    its (G, M) steering vectors; the maps are beamformerFreq('custom', ...) and the peak's vector is row
    xi_max of the same matrix (the object's steer_vector(f, xi_max))."""
    M = csm.shape[-1]
    normfactor = sig_loss_norm(r_diag, M, r_diag_norm)
    J = M * 2 if not n_iter else n_iter
    powers = np.zeros(J, 'd')
    res = None
    for i in ind:
        sv = np.ascontiguousarray(steer_vectors(freqs[i]), dtype=np.complex128)
        G = sv.shape[0]
        if out is None:
            out = np.zeros((csm.shape[0], G))
        if res is None:
            res = np.zeros(G, 'f')
        cs = np.array(csm[i], dtype='complex128', copy=True)
        h = beamformer_freq_custom(r_diag, normfactor, sv, csm=cs)[0]
        res *= 0.0
        for j in range(J):
            xi_max = h.argmax()
            powers[j] = hmax = h[xi_max]
            res[xi_max] += damp * hmax
            if j > stopn and hmax > powers[j - stopn]:
                break
            wmax = (sv[xi_max:xi_max + 1] * np.sqrt(normfactor))[0].conj()
            hh = wmax.copy()
            D1 = np.dot(cs.T - np.diag(np.diag(cs)), wmax) / hmax
            ww = wmax.conj() * wmax
            for _ in range(20):
                H = hh.conj() * hh
                hh = (D1 + H * wmax) / np.sqrt(1 + np.dot(ww, H))
            hh = hh[:, np.newaxis]
            csm1 = hmax * (hh * hh.conj().T)
            h1 = beamformer_freq_custom(r_diag, normfactor, sv, eig=(np.array((hmax,)),
                                                                    np.ascontiguousarray(hh.conj())))[0]
            h -= damp * h1
            cs -= damp * csm1.T
        out[i] = res
    return out


# ----------------------------------------------------------------------------------------------
# Block-wise spectra generators (acoular/fprocess.py)
# ----------------------------------------------------------------------------------------------
def rfft_blocks(samples: np.ndarray, block_size: int, window: str, overlap: str, precision: str, scaling: str,
                num: int):
    """``RFFT.result`` (acoular/fprocess.py:128-181): blocks (n, num_freqs * M) of scaled spectra."""
    wind = WINDOWS[window](block_size)
    if scaling in ('none', 'energy'):
        svalue = 1 / np.sqrt(np.dot(wind, wind) / block_size)
    else:
        svalue = 1 / wind.sum()
    wind = wind[:, np.newaxis]
    M = samples.shape[1]
    nf = block_size // 2 + 1
    fftdata = np.zeros((num, M * nf), dtype=precision)
    j = 0
    for i, data in enumerate(source_windows(samples, block_size, OVERLAPS[overlap])):
        j = i % num
        d = sfft.rfft(data * wind, n=block_size, axis=0).astype(precision)
        if scaling in ('amplitude', 'energy'):
            d[1:-1] *= 2.0
        d *= svalue
        fftdata[j] = d.reshape(-1)
        if j == num - 1:
            yield fftdata.copy()
    if j < num - 1:
        yield fftdata[: j + 1].copy()


def power_scale(block_size: int, sample_freq: float, scaling: str, single_sided: bool) -> float:
    """``AutoPowerSpectra._get_scaling_value`` (acoular/fprocess.py:323-329)."""
    scale = 1 / block_size**2
    if single_sided:
        scale *= 2
    if scaling == 'psd':
        scale *= block_size * sample_freq
    return scale


def auto_power_blocks(blocks, scale: float, precision: str):
    """``AutoPowerSpectra.result`` (acoular/fprocess.py:331-366)."""
    for temp in blocks:
        yield ((temp * temp.conjugate()).real * scale).astype(precision)


def cross_power_blocks(blocks, num_freqs: int, num_mics: int, scale: float, precision: str):
    """``CrossPowerSpectra.result`` (acoular/fprocess.py:425-467), calc_mode 'full': the per-snapshot
    CSM from the calcCSM restatement, its conjugate lower triangle (diagonal once), times scale."""
    csm_upper = np.zeros((num_freqs, num_mics, num_mics), dtype=precision)
    for data in blocks:
        flat = np.zeros((data.shape[0], num_freqs * num_mics * num_mics), dtype=precision)
        for i in range(data.shape[0]):
            spec = np.ascontiguousarray(data[i].astype(precision).reshape(num_freqs, num_mics))
            calc_csm_upper(csm_upper, spec)
            lower = csm_upper.conj().transpose(0, 2, 1)
            for f in range(num_freqs):
                np.fill_diagonal(lower[f], 0)
            flat[i] = (lower + csm_upper).reshape(-1)
            csm_upper[...] = 0
        yield flat * scale


def calc_csm_upper(csm: np.ndarray, spec: np.ndarray) -> None:
    """``calcCSM`` (fastFuncs.py:19-58) for one snapshot, in the array's precision (C restatement)."""
    F, M = spec.shape
    if csm.dtype == np.complex64:
        lib().orc_calc_csm_c64(_fp(csm), _fp(spec), F, M)
    else:
        lib().orc_calc_csm_c128(_dp(csm), _dp(spec), F, M)


def sig_loss_norm(r_diag: bool, num_mics: int, r_diag_norm: float = 0.0) -> float:
    """acoular/fbeamform.py:438-451."""
    if not r_diag:
        return 1.0
    if r_diag_norm == 0.0:
        n = float(num_mics)
        return n / (n - 1)
    return r_diag_norm


def beamformer_calc(csm: np.ndarray, freqs: np.ndarray, ind, r0, rm, c: float, steer_type: str, r_diag: bool,
                    r_diag_norm: float = 0.0, out: np.ndarray | None = None):
    """``BeamformerBase._calc`` (acoular/fbeamform.py:475-510) for a plain ``SteeringVector``."""
    G, M = rm.shape
    if out is None:
        out = np.zeros((csm.shape[0], G))
    normfactor = sig_loss_norm(r_diag, M, r_diag_norm)
    for i in ind:
        c_i = np.array(csm[i], dtype='complex128')
        b = beamformer_freq(steer_type, r_diag, normfactor, r0, rm, 2 * np.pi * freqs[i] / c, c_i)[0]
        if r_diag:
            b[np.sign(b) < 0] = 0.0
        out[i] = b
    return out


def band_indices(freq: np.ndarray, f: float, num):
    """Bin range of ``synthetic`` (acoular/fbeamform.py:566-577); ``(ind1, ind2)``."""
    if isinstance(num, list):
        f1, f2 = num[0], num[-1]
    else:
        f1 = f * 2.0 ** (-0.5 / num)
        f2 = f * 2.0 ** (+0.5 / num)
    return int(np.searchsorted(freq, f1)), int(np.searchsorted(freq, f2))


def synthetic(result: np.ndarray, freq: np.ndarray, f: float, num=0, shape=None):
    """``BeamformerBase.synthetic`` band sum (acoular/fbeamform.py:512-593) over a full result."""
    if num == 0:
        ind = int(np.searchsorted(freq, f))
        h = np.zeros_like(result[0]) if ind >= len(freq) else result[ind]
    else:
        ind1, ind2 = band_indices(freq, f, num)
        h = np.zeros_like(result[0]) if ind1 == ind2 else np.sum(result[ind1:ind2], 0)
    return h if shape is None else h.reshape(shape)


def L_p(x):
    """acoular/fbeamform.py:2412-2429."""
    return 10 * np.log10(np.maximum(x / 4e-10, np.finfo(x.dtype).eps))
