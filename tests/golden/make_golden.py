"""Generate the golden fixtures in this folder by running the reference's own code.

Run once, in a container that holds the reference sources, with ``ACOULAR_REFERENCE`` naming the
reference checkout (the folder that contains the ``acoular`` package)::

    ACOULAR_REFERENCE=<path to the acoular checkout> python tests/golden/make_golden.py

The reference (Acoular 26.08) cannot be imported whole here (``traits``/``tables`` are absent), so
this script loads its numba kernel module ``acoular/fastFuncs.py`` (+ ``internal.py``) under a stub
package and executes the reference's own glue methods, extracted from the source by ``ast`` with
their decorators removed, bound to plain stand-in objects:

* ``BaseSpectra._get_source_data`` / ``fftfreq``      acoular/spectra.py:128-184
* ``PowerSpectra._get_num_blocks`` / ``calc_csm``     acoular/spectra.py:281-283, 366-416
* ``dist_mat`` (re-jitted ``njit(fastmath=True)``)    acoular/environments.py:65-103
* ``Environment.apparent_r``                          acoular/environments.py:202-238
* ``RectGrid`` / ``RectGrid3D`` ``_get_pos``          acoular/grids.py:350-358, 552-560
* ``BeamformerBase.sig_loss_norm`` / ``_calc`` / ``synthetic``   acoular/fbeamform.py:438-593
* ``PowerSpectra._get__evd`` (np.linalg.eigh per bin)  acoular/spectra.py:351-364
* ``BeamformerEig._get_na`` / ``_calc``, ``BeamformerMusic._calc``   acoular/fbeamform.py:844-888, 911-944
* ``UniformFlowEnvironment.apparent_r``               acoular/environments.py:290-332
* ``SteeringVector._steer_funcs_freq`` (as source text) acoular/fbeamform.py:145-153
* ``PointSpreadFunction._psf_call``, ``BeamformerDamas._calc``   acoular/fbeamform.py:1096-1125, 1167-1208
* ``BeamformerFunctional._calc``, ``BeamformerOrth._calc``, ``BeamformerCleansc._calc`` (also with a
  custom steering object), ``SteeringVector.transfer`` / ``steer_vector``   acoular/fbeamform.py:712-786,
  1366-1490, 207-258
* ``RFFT.result`` / ``_scale``, ``AutoPowerSpectra._get_scaling_value`` / ``result``,
  ``CrossPowerSpectra.result``                        acoular/fprocess.py:35-181, 286-467
* ``SlotJet.v``, ``OpenJet.v``, ``RotatingFlow.v``, ``spiral_sphere``, ``GeneralFlowEnvironment.apparent_r`` /
  ``get_interpolator``                               acoular/environments.py:404-462, 518-573, 637-682, 685-980
* ``WNoiseGenerator.signal``, ``SignalGenerator.usignal``, ``PointSource.result``,
  ``_fill_mic_signal_block``, ``Mixer.result``        (fixture time data)

Outputs (small ``.npz`` files) are committed; the tests never read the reference at run time.
"""

from __future__ import annotations

import ast
import importlib.util
import os
import sys
import types
import warnings
from pathlib import Path
from types import SimpleNamespace

import numba as nb
import numpy as np
import scipy.linalg as spla
from scipy import fft
from scipy.signal import resample

if 'ACOULAR_REFERENCE' not in os.environ:
    raise SystemExit('set ACOULAR_REFERENCE to the reference checkout (the folder holding the acoular package)')
REF = Path(os.environ['ACOULAR_REFERENCE'])
OUT = Path(__file__).resolve().parent
sys.path.insert(0, str(OUT.parent.parent))


def _load_module(name):
    pkg = sys.modules.get('acoular')
    if pkg is None:
        pkg = types.ModuleType('acoular')
        pkg.__path__ = [str(REF / 'acoular')]
        sys.modules['acoular'] = pkg
    spec = importlib.util.spec_from_file_location(f'acoular.{name}', REF / 'acoular' / f'{name}.py')
    mod = importlib.util.module_from_spec(spec)
    sys.modules[f'acoular.{name}'] = mod
    spec.loader.exec_module(mod)
    return mod


internal = _load_module('internal')
fastFuncs = _load_module('fastFuncs')


def _extract(relpath, qualname, ns, rename=None):
    """Exec the source of ``Class.method`` or ``function`` from the reference, decorators removed."""
    src = (REF / relpath).read_text()
    tree = ast.parse(src)
    parts = qualname.split('.')
    body = tree.body
    node = None
    for p in parts:
        node = next(n for n in body if isinstance(n, (ast.ClassDef, ast.FunctionDef)) and n.name == p)
        body = node.body
    node.decorator_list = []
    if rename:
        node.name = rename
    mod = ast.Module(body=[node], type_ignores=[])
    code = compile(ast.fix_missing_locations(mod), f'{relpath}:{qualname}', 'exec')
    exec(code, ns)
    return ns[node.name]


NS = {'np': np, 'fft': fft, 'nb': nb, 'spla': spla, 'resample': resample, '_warn': warnings.warn,
      'calcCSM': fastFuncs.calcCSM, 'beamformerFreq': fastFuncs.beamformerFreq,
      'calcTransfer': fastFuncs.calcTransfer}

dist_mat_py = _extract('acoular/environments.py', 'dist_mat', NS)
dist_mat = nb.njit(fastmath=True)(dist_mat_py)
NS['dist_mat'] = dist_mat
apparent_r = _extract('acoular/environments.py', 'Environment.apparent_r', NS)
rect_get_pos = _extract('acoular/grids.py', 'RectGrid._get_pos', NS, rename='rect_get_pos')
rect3d_get_pos = _extract('acoular/grids.py', 'RectGrid3D._get_pos', NS, rename='rect3d_get_pos')
get_source_data = _extract('acoular/spectra.py', 'BaseSpectra._get_source_data', NS)
fftfreq_m = _extract('acoular/spectra.py', 'BaseSpectra.fftfreq', NS)
get_num_blocks = _extract('acoular/spectra.py', 'PowerSpectra._get_num_blocks', NS)
calc_csm = _extract('acoular/spectra.py', 'PowerSpectra.calc_csm', NS)
sig_loss_norm = _extract('acoular/fbeamform.py', 'BeamformerBase.sig_loss_norm', NS)
bf_calc = _extract('acoular/fbeamform.py', 'BeamformerBase._calc', NS)
synthetic = _extract('acoular/fbeamform.py', 'BeamformerBase.synthetic', NS)
get_evd = _extract('acoular/spectra.py', 'PowerSpectra._get__evd', NS)
eig_get_na = _extract('acoular/fbeamform.py', 'BeamformerEig._get_na', NS)
eig_calc = _extract('acoular/fbeamform.py', 'BeamformerEig._calc', NS, rename='eig_calc')
music_calc = _extract('acoular/fbeamform.py', 'BeamformerMusic._calc', NS, rename='music_calc')
uflow_apparent_r = _extract('acoular/environments.py', 'UniformFlowEnvironment.apparent_r', NS,
                            rename='uflow_apparent_r')
NS['calcPointSpreadFunction'] = fastFuncs.calcPointSpreadFunction
NS['damasSolverGaussSeidel'] = fastFuncs.damasSolverGaussSeidel
psf_call = _extract('acoular/fbeamform.py', 'PointSpreadFunction._psf_call', NS, rename='psf_call')
damas_calc = _extract('acoular/fbeamform.py', 'BeamformerDamas._calc', NS, rename='damas_calc')
functional_calc = _extract('acoular/fbeamform.py', 'BeamformerFunctional._calc', NS, rename='functional_calc')
orth_calc = _extract('acoular/fbeamform.py', 'BeamformerOrth._calc', NS, rename='orth_calc')
cleansc_calc = _extract('acoular/fbeamform.py', 'BeamformerCleansc._calc', NS, rename='cleansc_calc')
sv_transfer = _extract('acoular/fbeamform.py', 'SteeringVector.transfer', NS, rename='sv_transfer')
sv_steer_vector = _extract('acoular/fbeamform.py', 'SteeringVector.steer_vector', NS, rename='sv_steer_vector')
rfft_result = _extract('acoular/fprocess.py', 'RFFT.result', NS, rename='rfft_result')
rfft_scale = _extract('acoular/fprocess.py', 'RFFT._scale', NS, rename='rfft_scale')
aps_scaling = _extract('acoular/fprocess.py', 'AutoPowerSpectra._get_scaling_value', NS, rename='aps_scaling')
aps_result = _extract('acoular/fprocess.py', 'AutoPowerSpectra.result', NS, rename='aps_result')
cps_result = _extract('acoular/fprocess.py', 'CrossPowerSpectra.result', NS, rename='cps_result')
from scipy.integrate import ode as _ode  # noqa: E402
from scipy.interpolate import LinearNDInterpolator as _LNI  # noqa: E402
from scipy.spatial import ConvexHull as _CH  # noqa: E402
NS.update(ode=_ode, LinearNDInterpolator=_LNI, ConvexHull=_CH)
spiral_sphere = _extract('acoular/environments.py', 'spiral_sphere', NS)
NS['spiral_sphere'] = spiral_sphere
openjet_v = _extract('acoular/environments.py', 'OpenJet.v', NS, rename='openjet_v')
slotjet_v = _extract('acoular/environments.py', 'SlotJet.v', NS, rename='slotjet_v')
rotflow_v = _extract('acoular/environments.py', 'RotatingFlow.v', NS, rename='rotflow_v')
gflow_apparent_r = _extract('acoular/environments.py', 'GeneralFlowEnvironment.apparent_r', NS,
                            rename='gflow_apparent_r')
gflow_interp = _extract('acoular/environments.py', 'GeneralFlowEnvironment.get_interpolator', NS,
                        rename='gflow_interp')


def _steer_funcs_freq():
    """The reference's frequency-domain steering formulas, evaluated from its class body's source."""
    src = (REF / 'acoular/fbeamform.py').read_text()
    cls = next(n for n in ast.parse(src).body if isinstance(n, ast.ClassDef) and n.name == 'SteeringVector')
    assign = next(n for n in cls.body if isinstance(n, ast.Assign) and n.targets[0].id == '_steer_funcs_freq')
    return eval(compile(ast.Expression(assign.value.args[0]), 'fbeamform.py:_steer_funcs_freq', 'eval'), {'np': np})
w_signal = _extract('acoular/signals.py', 'WNoiseGenerator.signal', NS)
usignal = _extract('acoular/signals.py', 'SignalGenerator.usignal', NS)
fill_py = _extract('acoular/sources.py', '_fill_mic_signal_block', NS)
NS['_fill_mic_signal_block'] = nb.njit(error_model='numpy')(fill_py)
ps_result = _extract('acoular/sources.py', 'PointSource.result', NS)
mixer_result = _extract('acoular/tprocess.py', 'Mixer.result', NS)

WINDOWS = {'Rectangular': np.ones, 'Hanning': np.hanning, 'Hamming': np.hamming, 'Bartlett': np.bartlett,
           'Blackman': np.blackman}
OVERLAPS = {'None': 1, '50%': 2, '75%': 4, '87.5%': 8}


# ---------------------------------------------------------------------------------------------- stand-ins
class Env(SimpleNamespace):
    def apparent_r(self, gpos, mpos=0.0):
        return apparent_r(self, gpos, mpos)


def make_rect_grid(x_min, x_max, y_min, y_max, z, increment):
    i = abs(increment)
    nx = round((abs(x_max - x_min) + i) / i)
    ny = round((abs(y_max - y_min) + i) / i)
    g = SimpleNamespace(x_min=x_min, x_max=x_max, y_min=y_min, y_max=y_max, z=z, increment=increment,
                        nxsteps=nx, nysteps=ny, size=nx * ny, shape=(nx, ny))
    g.pos = rect_get_pos(g)
    return g


def make_rect_grid3d(x_min, x_max, y_min, y_max, z_min, z_max, increment):
    i = abs(increment)
    nx = round((abs(x_max - x_min) + i) / i)
    ny = round((abs(y_max - y_min) + i) / i)
    nz = round((abs(z_max - z_min) + i) / i)
    g = SimpleNamespace(x_min=x_min, x_max=x_max, y_min=y_min, y_max=y_max, z_min=z_min, z_max=z_max,
                        nxsteps=nx, nysteps=ny, nzsteps=nz, size=nx * ny * nz, shape=(nx, ny, nz))
    g.pos = rect3d_get_pos(g)
    return g


class WNoise(SimpleNamespace):
    def signal(self):
        return w_signal(self)

    def usignal(self, factor):
        return usignal(self, factor)


class PSource(SimpleNamespace):
    def _validate_locations(self):
        pass

    def result(self, num=128):
        return ps_result(self, num)


class Mix(SimpleNamespace):
    def validate_sources(self):
        pass

    def result(self, num):
        return mixer_result(self, num)


class Samples(SimpleNamespace):
    def result(self, num=128):
        i = 0
        while i < self.num_samples:
            yield self.data[i:num + i]
            i += num


def reference_time_data(mpos, locs, seeds, rms, fs, nsamples, c=343.0, num=4096):
    env = Env(c=c)
    mics = SimpleNamespace(pos=mpos, num_mics=mpos.shape[1])
    srcs = []
    for loc, seed, r in zip(locs, seeds, rms):
        sig = WNoise(seed=seed, rms=r, num_samples=nsamples, sample_freq=fs)
        srcs.append(PSource(signal=sig, mics=mics, loc=np.asarray(loc, float).reshape(3, 1), env=env, start_t=0.0,
                            start=0.0, up=16, prepadding='loop', num_samples=nsamples, sample_freq=fs,
                            num_channels=mpos.shape[1]))
    mix = Mix(source=srcs[0], sources=srcs[1:])
    return np.concatenate([b.copy() for b in mix.result(num)])


def reference_csm(data, fs, block_size, window, overlap, precision):
    src = Samples(data=data, num_samples=data.shape[0], num_channels=data.shape[1], sample_freq=fs)
    ps = SimpleNamespace(source=src, block_size=block_size, window_=WINDOWS[window], overlap_=OVERLAPS[overlap],
                         precision=precision, num_channels=data.shape[1])
    ps._get_source_data = lambda: get_source_data(ps)
    ps.num_blocks = get_num_blocks(ps)
    return calc_csm(ps), fftfreq_m(ps)


class Steer(SimpleNamespace):
    pass


class PSFStandIn(SimpleNamespace):
    """PointSpreadFunction without its cache: ``psf`` is the 'full' branch of ``calc_psf``
    (acoular/fbeamform.py:1087-1089) cast to ``precision`` like its result array."""

    freq = 1.0

    def _psf_call(self, ind):
        return psf_call(self, ind)

    @property
    def psf(self):
        gs = self.steer.grid.size
        ac = np.zeros((gs, gs), dtype=self.precision)
        ac[:] = self._psf_call(np.arange(gs))
        return ac


NS['SteeringVector'] = Steer
NS['PointSpreadFunction'] = PSFStandIn


def reference_bf_result(csm, freqs, mpos, gpos, gshape, steer_type, r_diag, c=343.0, ref=None, r_diag_norm=0.0,
                        ind=None):
    """Run ``BeamformerBase._calc`` for bins ``ind`` (all if None); returns (F, G) and r0, rm."""
    env = Env(c=c)
    r0 = apparent_r(env, gpos) if ref is None else apparent_r(env, gpos, np.asarray(ref, float)[:, None])
    rm = np.atleast_2d(apparent_r(env, gpos, mpos))
    F, G = csm.shape[0], gpos.shape[1]
    bf = SimpleNamespace(_f=freqs, r_diag=r_diag, r_diag_norm=r_diag_norm,
                         freq_data=SimpleNamespace(num_channels=mpos.shape[1], csm=csm))
    bf.sig_loss_norm = lambda: sig_loss_norm(bf)
    bf._beamformer_params = lambda: (steer_type, lambda f: (r0, rm, 2 * np.pi * f / c))
    bf._ac = np.zeros((F, G))
    bf._fr = np.zeros(F, dtype='int8')
    bf_calc(bf, np.arange(F) if ind is None else np.asarray(ind))
    return bf._ac, r0, rm


def reference_synthetic(ac_full, freqs, gshape, f, num):
    bf = SimpleNamespace(result=ac_full, freq_data=SimpleNamespace(fftfreq=lambda: freqs),
                         steer=SimpleNamespace(grid=SimpleNamespace(shape=gshape)))
    NS['BeamformerAdaptiveGrid'] = type('BeamformerAdaptiveGrid', (), {})
    NS['BeamformerSODIX'] = type('BeamformerSODIX', (), {})
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        return synthetic(bf, f, num)


STEERS = ['classic', 'inverse', 'true level', 'true location']


def golden_env():
    """Environment.apparent_r on the reference's regression grid, checked against its committed array."""
    g = make_rect_grid3d(-0.2, 0.2, -0.2, 0.2, 0.5, 0.9, 0.2)
    mics = np.array(((0.5, 0.5, 0), (0, 0, 0), (-0.5, -0.5, 0)), dtype=float)
    env = Env(c=343.0)
    res_arr = np.vstack((apparent_r(env, g.pos, mics).T, apparent_r(env, g.pos).T))
    res_sc = np.vstack((apparent_r(env, g.pos, 0.0).T, apparent_r(env, g.pos).T))
    base = REF / 'tests/regression/_regtest_outputs'
    exp_arr = np.load(base / 'test_environments.test_environment[RectGrid3D-mics-arr-default-Environment]__0/arrays.npy')
    exp_sc = np.load(base / 'test_environments.test_environment[RectGrid3D-mics-scalar-default-Environment]__0/arrays.npy')
    np.testing.assert_allclose(res_arr, exp_arr, rtol=1e-5, atol=1e-8)
    np.testing.assert_allclose(res_sc, exp_sc, rtol=1e-5, atol=1e-8)
    np.savez_compressed(OUT / 'env_apparent_r.npz', gpos=g.pos, mpos=mics, mics_arr=exp_arr, mics_scalar=exp_sc,
                        rm_ref=apparent_r(env, g.pos, mics))
    print('env_apparent_r.npz: matches the reference regression arrays')


def golden_small():
    """8 mics, 2000 samples of three monopoles: CSMs for several spectra settings + all maps."""
    from acoular_b200.microphones import disk_mics
    mpos = disk_mics(8, 0.5, seed=7).pos
    fs = 51200.0
    data = reference_time_data(mpos, [(-0.1, -0.1, -0.3), (0.15, 0, -0.3), (0, 0.1, -0.3)], [1, 2, 3],
                               [1.0, 0.7, 0.5], fs, 2000)
    out = {'mpos': mpos, 'data': data, 'fs': fs}
    csm_cases = [(128, 'Hanning', '50%', 'complex128'), (256, 'Rectangular', 'None', 'complex128'),
                 (128, 'Blackman', '75%', 'complex64'), (256, 'Hamming', '87.5%', 'complex128'),
                 (128, 'Bartlett', '50%', 'complex64')]
    for i, (bs, win, ov, prec) in enumerate(csm_cases):
        csm, freqs = reference_csm(data, fs, bs, win, ov, prec)
        out[f'csm{i}'] = csm
        out[f'csm{i}_case'] = np.array([str(bs), win, ov, prec])
        out[f'freqs{i}'] = freqs
    g = make_rect_grid(-0.2, 0.2, -0.2, 0.2, -0.3, 0.05)
    out['gpos'] = g.pos
    out['gshape'] = np.array(g.shape)
    csm, freqs = out['csm0'], out['freqs0']
    ind = np.arange(10, 31)
    out['bins'] = ind
    for st in STEERS:
        for rd in (False, True):
            ac_full, r0, rm = reference_bf_result(csm, freqs, mpos, g.pos, g.shape, st, rd, ind=ind)
            key = f'map_{st.replace(" ", "_")}_{int(rd)}'
            out[key] = ac_full[ind]
            out['syn_' + key] = reference_synthetic(ac_full, freqs, g.shape, 8000.0, 3)
    # a non-origin reference position and a user r_diag_norm
    ac_full, r0, _ = reference_bf_result(csm, freqs, mpos, g.pos, g.shape, 'true level', True,
                                         ref=(0.1, -0.05, 0.02), r_diag_norm=1.25, ind=ind)
    out['map_ref_rdn'] = ac_full[ind]
    out['r0_ref'] = r0
    np.savez_compressed(OUT / 'small_kat.npz', **out)
    print('small_kat.npz written')


def golden_rank1():
    """Rank-1 CSM of one monopole (the reference's integrate test set-up, tests/unittests/test_integrate.py)."""
    rng1 = np.random.RandomState(1)
    mpos = rng1.normal(size=3 * 5).reshape((3, 5))
    f = 2000.0
    src = np.array([[0.0], [0.0], [1.0]])
    env = Env(c=343.0)
    r0 = apparent_r(env, src)
    rm = np.atleast_2d(apparent_r(env, src, mpos))
    transf = fastFuncs.calcTransfer(r0, rm, np.array(2 * np.pi * f / 343.0))
    csm = (transf.T @ transf.T.conj().T)[None]  # (1, M, M)
    g = make_rect_grid(-0.5, 0.5, -0.5, 0.5, 1.0, 0.25)
    out = {'mpos': mpos, 'csm': csm, 'freqs': np.array([f]), 'gpos': g.pos, 'gshape': np.array(g.shape)}
    for st in STEERS:
        for rd in (False, True):
            ac_full, _, _ = reference_bf_result(csm, np.array([f]), mpos, g.pos, g.shape, st, rd)
            out[f'map_{st.replace(" ", "_")}_{int(rd)}'] = ac_full[0]
    np.savez_compressed(OUT / 'rank1_kat.npz', **out)
    print('rank1_kat.npz written')


def golden_config1():
    """The 64-mic three-source workload: CSM bins of the 8 kHz third-octave band and all 8 maps."""
    from acoular_b200 import workloads
    wl = workloads.three_sources_64()
    data_ref = reference_time_data(wl.mics.pos, wl.locs, wl.seeds, wl.rms, wl.fs, wl.num_samples)
    data_ours = wl.time_data()
    diff = np.abs(data_ref - data_ours).max() / np.abs(data_ref).max()
    print('config1 time data: restated generator vs reference max rel diff', diff)
    assert diff < 1e-12
    csm, freqs = reference_csm(data_ref, wl.fs, 128, 'Hanning', '50%', 'complex128')
    g = wl.grid
    out = {'freqs': freqs, 'band_bins': np.arange(18, 23), 'csm_band': csm[18:23],
           'csm_diag': np.real(np.einsum('fmm->fm', csm)), 'csm_sum': csm.sum(axis=(1, 2)),
           'data_stats': np.array([data_ref.sum(), (data_ref ** 2).sum(), data_ref[::997, ::7].sum()])}
    for st in STEERS:
        for rd in (False, True):
            ac_full, _, _ = reference_bf_result(csm, freqs, wl.mics.pos, g.pos, g.shape, st, rd,
                                                ind=np.arange(18, 23))
            key = f'map_{st.replace(" ", "_")}_{int(rd)}'
            out[key] = ac_full[18:23]
            out['syn_' + key] = reference_synthetic(ac_full, freqs, g.shape, 8000.0, 3)
    np.savez_compressed(OUT / 'config1_band.npz', **out)
    print('config1_band.npz written')


def reference_eig_result(kind, csm, freqs, mpos, gpos, steer_type, r_diag, n, ind, c=343.0, r_diag_norm=0.0):
    """``BeamformerEig._calc`` / ``BeamformerMusic._calc`` for bins ``ind`` with the reference's eigh."""
    env = Env(c=c)
    r0 = apparent_r(env, gpos)
    rm = np.atleast_2d(apparent_r(env, gpos, mpos))
    M = mpos.shape[1]
    eva, eve = get_evd(SimpleNamespace(precision='complex128', csm=csm))
    bf = SimpleNamespace(_f=freqs, r_diag=r_diag, r_diag_norm=r_diag_norm, n=n,
                         steer=SimpleNamespace(mics=SimpleNamespace(num_mics=M)),
                         freq_data=SimpleNamespace(num_channels=M, eigvals=eva, eigvecs=eve))
    bf.na = eig_get_na(bf)
    bf.sig_loss_norm = lambda: sig_loss_norm(bf)
    bf._beamformer_params = lambda: (steer_type, lambda f: (r0, rm, 2 * np.pi * f / c))
    bf._ac = np.zeros((csm.shape[0], gpos.shape[1]))
    bf._fr = np.zeros(csm.shape[0], dtype='int8')
    (eig_calc if kind == 'eig' else music_calc)(bf, np.asarray(ind))
    return bf._ac[ind], eva[ind], eve[ind], bf.na


def golden_eig():
    """Eigenvalue beamformers (BeamformerEig for several components, BeamformerMusic) on the 8-mic
    CSM of small_kat.npz and the 64-mic config-1 band, with the reference's own eigendecomposition."""
    small = np.load(OUT / 'small_kat.npz')
    out = {}
    cases = [('s', small['csm0'], small['freqs0'], small['mpos'], small['gpos'], np.arange(10, 31))]
    from acoular_b200 import workloads
    wl = workloads.three_sources_64()
    data_ref = reference_time_data(wl.mics.pos, wl.locs, wl.seeds, wl.rms, wl.fs, wl.num_samples)
    csm64, freqs64 = reference_csm(data_ref, wl.fs, 128, 'Hanning', '50%', 'complex128')
    cases.append(('c1', csm64, freqs64, wl.mics.pos, wl.grid.pos, np.arange(18, 23)))
    for tag, csm, freqs, mpos, gpos, ind in cases:
        M = mpos.shape[1]
        out[f'{tag}_mpos'], out[f'{tag}_gpos'], out[f'{tag}_bins'] = mpos, gpos, ind
        out[f'{tag}_freqs'] = freqs[ind]
        first = True
        for n in (-1, 0, M // 2):
            for st in STEERS:
                for rd in (False, True):
                    res, eva, eve, na = reference_eig_result('eig', csm, freqs, mpos, gpos, st, rd, n, ind)
                    out[f'{tag}_eig_n{n}_{st.replace(" ", "_")}_{int(rd)}'] = res
                    out[f'{tag}_eig_n{n}_na'] = np.array(na)
                    if first:
                        out[f'{tag}_eigvals'], out[f'{tag}_eigvecs'] = eva, eve
                        first = False
        for n in (1, 3):
            for st in STEERS:
                res, _, _, na = reference_eig_result('music', csm, freqs, mpos, gpos, st, False, n, ind,
                                                     r_diag_norm=1.0)
                out[f'{tag}_music_n{n}_{st.replace(" ", "_")}'] = res
                out[f'{tag}_music_n{n}_na'] = np.array(na)
    np.savez_compressed(OUT / 'eig_kat.npz', **out)
    print('eig_kat.npz written', len(out), 'arrays')


def golden_custom_flow():
    """Custom steering vectors (beamformerFreq('custom', ...), full / removed diagonal / eigen) and
    the uniform-flow environment on the 8-mic case of small_kat.npz."""
    small = np.load(OUT / 'small_kat.npz')
    csm, freqs, mpos, gpos = small['csm0'], small['freqs0'], small['mpos'], small['gpos']
    M = mpos.shape[1]
    env = Env(c=343.0)
    r0, rm = apparent_r(env, gpos), np.atleast_2d(apparent_r(env, gpos, mpos))
    funcs = _steer_funcs_freq()
    eva, eve = get_evd(SimpleNamespace(precision='complex128', csm=csm))
    out = {'bins': np.array([10, 20])}
    for b in out['bins']:
        k = 2 * np.pi * freqs[b] / 343.0
        trans = fastFuncs.calcTransfer(r0, rm, np.array(k))
        out[f'trans_{b}'] = trans
        for st in STEERS:
            h = np.ascontiguousarray(funcs[st](trans))
            out[f'steer_{st.replace(" ", "_")}_{b}'] = h
            for rd in (False, True):
                res, nrm = fastFuncs.beamformerFreq('custom', rd, 1.25, h, np.ascontiguousarray(csm[b]))
                out[f'cust_{st.replace(" ", "_")}_{int(rd)}_{b}'] = res
                out[f'custn_{st.replace(" ", "_")}_{int(rd)}_{b}'] = nrm
                res, nrm = fastFuncs.beamformerFreq('custom', rd, 1.25, h,
                                                    (np.array(eva[b, M - 2:]), np.ascontiguousarray(eve[b][:, M - 2:])))
                out[f'custe_{st.replace(" ", "_")}_{int(rd)}_{b}'] = res
    out['eigvals'], out['eigvecs'] = eva[out['bins']], eve[out['bins']]
    # uniform flow: Mach 0.3 along (1, 0.5, 0); the fast path of BeamformerBase._calc with its distances
    fl = SimpleNamespace(ma=0.3, fdv=np.array((1.0, 0.5, 0.0)))
    r0f, rmf = uflow_apparent_r(fl, gpos), np.atleast_2d(uflow_apparent_r(fl, gpos, mpos))
    out['flow_r0'], out['flow_rm'] = r0f, rmf
    ind = np.arange(10, 31)
    for st in STEERS:
        for rd in (False, True):
            bf = SimpleNamespace(_f=freqs, r_diag=rd, r_diag_norm=0.0,
                                 freq_data=SimpleNamespace(num_channels=M, csm=csm))
            bf.sig_loss_norm = lambda bf=bf: sig_loss_norm(bf)
            bf._beamformer_params = lambda st=st: (st, lambda f: (r0f, rmf, 2 * np.pi * f / 343.0))
            bf._ac = np.zeros((csm.shape[0], gpos.shape[1]))
            bf._fr = np.zeros(csm.shape[0], dtype='int8')
            bf_calc(bf, ind)
            out[f'flow_{st.replace(" ", "_")}_{int(rd)}'] = bf._ac[ind]
    np.savez_compressed(OUT / 'custom_flow_kat.npz', **out)
    print('custom_flow_kat.npz written', len(out), 'arrays')


def reference_damas_result(csm, freqs, r0, rm, steer_type, r_diag, n_iter, damp, psf_precision, ind, c=343.0):
    """``BeamformerDamas._calc`` for bins ``ind`` with the reference's PSF and Gauss-Seidel kernels."""
    G, M = rm.shape
    steer = Steer(steer_type=steer_type, r0=r0, rm=rm, env=SimpleNamespace(c=c), grid=SimpleNamespace(size=G))
    bf = SimpleNamespace(_f=freqs, r_diag=r_diag, r_diag_norm=0.0, n_iter=n_iter, damp=damp,
                         psf_precision=psf_precision, calcmode='full', cached=False, steer=steer,
                         freq_data=SimpleNamespace(num_channels=M, csm=csm))
    bf.sig_loss_norm = lambda: sig_loss_norm(bf)
    bf._beamformer_params = lambda: (steer_type, lambda f: (r0, rm, 2 * np.pi * f / c))
    bf._ac = np.zeros((csm.shape[0], G))
    bf._fr = np.zeros(csm.shape[0], dtype='int8')
    damas_calc(bf, np.asarray(ind))
    return bf._ac[ind]


def golden_psf_damas():
    """PointSpreadFunction._psf_call (full and selected sources, free field and uniform flow) and
    BeamformerDamas._calc on the 8-mic case of small_kat.npz and two bins of the 64-mic band."""
    small = np.load(OUT / 'small_kat.npz')
    csm, freqs, mpos, gpos = small['csm0'], small['freqs0'], small['mpos'], small['gpos']
    env = Env(c=343.0)
    r0, rm = apparent_r(env, gpos), np.atleast_2d(apparent_r(env, gpos, mpos))
    G = gpos.shape[1]
    out = {'bins': np.array([12, 20, 28]), 'psf_bin': np.array(20), 'src': np.array([3, 40, 77])}
    for st in STEERS:
        key = st.replace(' ', '_')
        p = PSFStandIn(steer=Steer(steer_type=st, r0=r0, rm=rm, env=env, grid=SimpleNamespace(size=G)),
                       calcmode='full', precision='float64', cached=False)
        p.freq = freqs[20]
        out[f'psf_full_{key}'] = p.psf
        p.precision = 'float32'
        out[f'psf_full32_{key}'] = p.psf
        out[f'psf_src_{key}'] = p._psf_call(out['src'])
        for rd in (False, True):
            out[f'damas_{key}_{int(rd)}'] = reference_damas_result(csm, freqs, r0, rm, st, rd, 10, 0.98, 'float64',
                                                                   out['bins'])
    out['damas_default_classic_0'] = reference_damas_result(csm, freqs, r0, rm, 'classic', False, 100, 1.0,
                                                            'float64', out['bins'])
    out['damas_f32_true_level_1'] = reference_damas_result(csm, freqs, r0, rm, 'true level', True, 10, 0.98,
                                                           'float32', out['bins'])
    fl = SimpleNamespace(ma=0.3, fdv=np.array((1.0, 0.5, 0.0)))
    r0f, rmf = uflow_apparent_r(fl, gpos), np.atleast_2d(uflow_apparent_r(fl, gpos, mpos))
    for st in STEERS:
        p = PSFStandIn(steer=Steer(steer_type=st, r0=r0f, rm=rmf, env=env, grid=SimpleNamespace(size=G)),
                       calcmode='block', precision='float64', cached=False)
        p.freq = freqs[20]
        out[f'psf_flow_{st.replace(" ", "_")}'] = p._psf_call(out['src'])
    out['flow_r0'], out['flow_rm'] = r0f, rmf
    from acoular_b200 import workloads
    wl = workloads.three_sources_64()
    data_ref = reference_time_data(wl.mics.pos, wl.locs, wl.seeds, wl.rms, wl.fs, wl.num_samples)
    csm64, freqs64 = reference_csm(data_ref, wl.fs, 128, 'Hanning', '50%', 'complex128')
    r064 = apparent_r(env, wl.grid.pos)
    rm64 = np.atleast_2d(apparent_r(env, wl.grid.pos, wl.mics.pos))
    out['c1_bins'] = np.array([18, 21])
    for st, rd in (('classic', False), ('true level', True)):
        out[f'c1_damas_{st.replace(" ", "_")}_{int(rd)}'] = reference_damas_result(
            csm64, freqs64, r064, rm64, st, rd, 10, 0.98, 'float64', out['c1_bins'])
    np.savez_compressed(OUT / 'psf_damas_kat.npz', **out)
    print('psf_damas_kat.npz written', len(out), 'arrays')


class SteerFull(SimpleNamespace):
    """SteeringVector stand-in with the reference's transfer / steer_vector (fbeamform.py:207-258)."""

    def transfer(self, f, ind=None):
        return sv_transfer(self, f, ind)

    def steer_vector(self, f, ind=None):
        return sv_steer_vector(self, f, ind)


def _eig_bf(csm, freqs, mpos, gpos, steer_type, r_diag, c=343.0, r_diag_norm=0.0, **kw):
    env = Env(c=c)
    r0, rm = apparent_r(env, gpos), np.atleast_2d(apparent_r(env, gpos, mpos))
    M = mpos.shape[1]
    eva, eve = get_evd(SimpleNamespace(precision='complex128', csm=csm))
    steer = SteerFull(steer_type=steer_type, r0=r0, rm=rm, env=env, _steer_funcs_freq=_steer_funcs_freq(),
                      grid=SimpleNamespace(size=gpos.shape[1]), mics=SimpleNamespace(num_mics=M))
    bf = SimpleNamespace(_f=freqs, r_diag=r_diag, r_diag_norm=r_diag_norm, steer=steer,
                         freq_data=SimpleNamespace(num_channels=M, csm=csm, eigvals=eva, eigvecs=eve), **kw)
    bf.sig_loss_norm = lambda: sig_loss_norm(bf)
    bf._beamformer_params = lambda: (steer_type, lambda f: (r0, rm, 2 * np.pi * f / c))
    bf._ac = np.zeros((csm.shape[0], gpos.shape[1]))
    bf._fr = np.zeros(csm.shape[0], dtype='int8')
    return bf


def golden_functional_orth_cleansc():
    """BeamformerFunctional, BeamformerOrth and BeamformerCleansc (fbeamform.py:688-790, 1333-1492) on the
    8-mic case of small_kat.npz and the 64-mic band, with the reference's own eigh, transfer and kernels."""
    small = np.load(OUT / 'small_kat.npz')
    cases = [('s', small['csm0'], small['freqs0'], small['mpos'], small['gpos'], np.array([12, 20, 28]))]
    from acoular_b200 import workloads
    wl = workloads.three_sources_64()
    data_ref = reference_time_data(wl.mics.pos, wl.locs, wl.seeds, wl.rms, wl.fs, wl.num_samples)
    csm64, freqs64 = reference_csm(data_ref, wl.fs, 128, 'Hanning', '50%', 'complex128')
    cases.append(('c1', csm64, freqs64, wl.mics.pos, wl.grid.pos, np.array([18, 21])))
    out = {}
    for tag, csm, freqs, mpos, gpos, ind in cases:
        out[f'{tag}_bins'] = ind
        M = mpos.shape[1]
        for st in STEERS:
            key = st.replace(' ', '_')
            for gamma in (1.0, 3.0):
                bf = _eig_bf(csm, freqs, mpos, gpos, st, False, r_diag_norm=1.0, gamma=gamma)
                functional_calc(bf, ind)
                out[f'{tag}_functional_{key}_g{gamma:g}'] = bf._ac[ind]
            for rd in (False, True):
                for eva_list in ([-1], [-1, -2, -3], [M - 6, 2]):
                    bf = _eig_bf(csm, freqs, mpos, gpos, st, rd, eva_list=np.array(eva_list))
                    orth_calc(bf, ind)
                    out[f'{tag}_orth_{key}_{int(rd)}_{"_".join(str(e) for e in eva_list)}'] = bf._ac[ind]
            for rd in (False, True):
                for n_iter, damp, stopn in ((0, 0.6, 3), (10, 0.9, 4)):
                    bf = _eig_bf(csm, freqs, mpos, gpos, st, rd, n_iter=n_iter, damp=damp, stopn=stopn)
                    cleansc_calc(bf, ind)
                    out[f'{tag}_cleansc_{key}_{int(rd)}_{n_iter}_{damp:g}_{stopn}'] = bf._ac[ind]
    np.savez_compressed(OUT / 'functional_orth_cleansc_kat.npz', **out)
    print('functional_orth_cleansc_kat.npz written', len(out), 'arrays')


class SteerShaded(SteerFull):
    """A steering object of its own (a SteeringVector subclass): the reference's steer_vector shaded by a
    per-mic weight; BeamformerCleansc routes it through the custom-steering kernels."""

    def steer_vector(self, f, ind=None):
        return sv_steer_vector(self, f, ind) * self.shade[np.newaxis, :]


def cleansc_shade(M):
    """Per-mic shading of the custom steering object in cleansc_custom_kat.npz (a Hann taper over the mics)."""
    return 0.5 + 0.5 * np.cos(np.pi * (np.arange(M) - (M - 1) / 2) / M)


def golden_cleansc_custom():
    """BeamformerCleansc._calc (fbeamform.py:1424-1490) with a steering object other than the plain
    SteeringVector: _beamformer_params gives ('custom', steer.steer_vector) (fbeamform.py:470-472), so the
    maps use beamformerFreq('custom', ...) and the peak's vector is the object's steer_vector(f, xi)."""
    small = np.load(OUT / 'small_kat.npz')
    csm, freqs, mpos, gpos = small['csm0'], small['freqs0'], small['mpos'], small['gpos']
    ind = np.array([12, 20, 28])
    out = {'bins': ind}
    env = Env(c=343.0)
    r0, rm = apparent_r(env, gpos), np.atleast_2d(apparent_r(env, gpos, mpos))
    M = mpos.shape[1]
    for st in ('true level', 'classic'):
        steer = SteerShaded(steer_type=st, r0=r0, rm=rm, env=env, _steer_funcs_freq=_steer_funcs_freq(),
                            grid=SimpleNamespace(size=gpos.shape[1]), mics=SimpleNamespace(num_mics=M),
                            shade=cleansc_shade(M))
        for rd in (False, True):
            for n_iter, damp, stopn in ((0, 0.6, 3), (10, 0.9, 4)):
                bf = SimpleNamespace(_f=freqs, r_diag=rd, r_diag_norm=0.0, steer=steer, n_iter=n_iter, damp=damp,
                                     stopn=stopn, freq_data=SimpleNamespace(num_channels=M, csm=csm))
                bf.sig_loss_norm = lambda bf=bf: sig_loss_norm(bf)
                bf._beamformer_params = lambda steer=steer: ('custom', steer.steer_vector)
                bf._ac = np.zeros((csm.shape[0], gpos.shape[1]))
                bf._fr = np.zeros(csm.shape[0], dtype='int8')
                cleansc_calc(bf, ind)
                out[f'{st.replace(" ", "_")}_{int(rd)}_{n_iter}_{damp:g}_{stopn}'] = bf._ac[ind]
    np.savez_compressed(OUT / 'cleansc_custom_kat.npz', **out)
    print('cleansc_custom_kat.npz written', len(out), 'arrays')


class RfftStandIn(SimpleNamespace):
    """RFFT (fprocess.py:35-181) over a Samples source, with the reference's generator and scaling."""

    def _get_source_data(self):
        return get_source_data(self)

    def _scale(self, data, scaling_value):
        return rfft_scale(self, data, scaling_value)

    def result(self, num=1):
        return rfft_result(self, num)


class ApsStandIn(SimpleNamespace):
    def _get_scaling_value(self):
        return aps_scaling(self)

    def result(self, num=1):
        return (cps_result if hasattr(self, 'calc_mode') else aps_result)(self, num)


def golden_fprocess():
    """RFFT / AutoPowerSpectra / CrossPowerSpectra generators (fprocess.py:35-467) on the 8-mic time data
    of small_kat.npz: every scaling, both precisions, overlaps and block counts that leave a short last
    block."""
    small = np.load(OUT / 'small_kat.npz')
    data, fs = small['data'], float(small['fs'])
    out = {}
    cases = [(128, 'Hanning', '50%', 'complex128', 'none', 7), (256, 'Rectangular', 'None', 'complex128', 'energy', 3),
             (64, 'Blackman', '75%', 'complex64', 'amplitude', 16), (128, 'Hamming', 'None', 'complex64', 'none', 4)]
    for ci, (bs, win, ov, prec, scaling, num) in enumerate(cases):
        src = Samples(data=data, num_samples=data.shape[0], num_channels=data.shape[1], sample_freq=fs)
        rf = RfftStandIn(source=src, block_size=bs, window_=WINDOWS[win], overlap_=OVERLAPS[ov], precision=prec,
                         scaling=scaling, workers=None, num_channels=data.shape[1], num_freqs=bs // 2 + 1,
                         sample_freq=fs)
        blocks = [b.copy() for b in rf.result(num)]
        out[f'rfft{ci}_case'] = np.array([str(bs), win, ov, prec, scaling, str(num)])
        out[f'rfft{ci}_sizes'] = np.array([b.shape[0] for b in blocks])
        out[f'rfft{ci}'] = np.concatenate(blocks)
        for ai, (sc, ss, ap) in enumerate([('power', True, 'float64'), ('psd', False, 'float32')]):
            aps = ApsStandIn(source=rf, scaling=sc, single_sided=ss, precision=ap, block_size=bs, num_freqs=bs // 2 + 1,
                             num_channels=data.shape[1])
            out[f'aps{ci}_{ai}'] = np.concatenate([b.copy() for b in aps.result(num)])
        cprec = 'complex64' if prec == 'complex64' else 'complex128'
        cps = ApsStandIn(source=rf, scaling='psd' if ci % 2 else 'power', single_sided=True, precision=cprec,
                         block_size=bs, num_freqs=bs // 2 + 1, num_channels=data.shape[1] ** 2, calc_mode='full')
        blocks = [b.copy() for b in cps.result(num)]
        allc = np.concatenate(blocks)
        out[f'cps{ci}'] = allc[:2 * num]                      # the first two blocks in full
        out[f'cps{ci}_sum'] = allc.astype(np.complex128).sum(axis=0)   # and a sum over every snapshot
        out[f'cps{ci}_sizes'] = np.array([b.shape[0] for b in blocks])
    np.savez_compressed(OUT / 'fprocess_kat.npz', **out)
    print('fprocess_kat.npz written', len(out), 'arrays')


def golden_general_flow():
    """The flow fields' v() and GeneralFlowEnvironment.apparent_r (ray tracing, acoular/environments.py:335-980)
    for an open jet, a slot jet and a rotating flow on a small grid and 3 microphones."""
    rng = np.random.RandomState(5)
    pts = rng.uniform(-0.5, 0.5, (12, 3)) + np.array((0.6, 0.0, 0.4))
    fields = {
        'openjet': (SimpleNamespace(v0=20.0, origin=np.zeros(3), D=0.4, l=6.2), openjet_v),
        'slotjet': (SimpleNamespace(v0=15.0, origin=np.zeros(3), flow=np.array((1.0, 0.0, 0.0)),
                                    plane=np.array((0.0, 1.0, 0.0)), B=0.3, l=5.2), slotjet_v),
        'rotating': (SimpleNamespace(rps=2.0, v0=3.0, origin=np.zeros(3), omega=2 * np.pi * 2.0), rotflow_v),
    }
    out = {'pts': pts}
    for name, (ff, vfun) in fields.items():
        vs, js = zip(*[vfun(ff, p) for p in pts])
        out[f'{name}_v'], out[f'{name}_jac'] = np.array(vs), np.array(js)
    g = make_rect_grid(-0.2, 0.2, -0.2, 0.2, 0.6, 0.2)
    mpos = np.array(((0.3, -0.2, 0.0), (-0.25, 0.1, 0.0), (0.0, 0.3, 0.05)))
    out['gpos'], out['mpos'] = g.pos, mpos
    for name, (ff, vfun) in fields.items():
        ffo = SimpleNamespace(**vars(ff))
        ffo.v = lambda x, ff=ff, vfun=vfun: vfun(ff, x)
        env = SimpleNamespace(c=343.0, ff=ffo, N=64, Om=np.pi, roi=None, idict={})
        env.get_interpolator = lambda roi, x0, env=env: gflow_interp(env, roi, x0)
        out[f'{name}_rm'] = gflow_apparent_r(env, g.pos, mpos)
        out[f'{name}_r0'] = gflow_apparent_r(env, g.pos)
    out['sphere'] = spiral_sphere(40, np.pi, b=np.array((0.3, -0.5, 1.0)))
    np.savez_compressed(OUT / 'general_flow_kat.npz', **out)
    print('general_flow_kat.npz written', len(out), 'arrays')


if __name__ == '__main__':
    if os.environ.get('ACB_GOLDEN_ONLY') == 'general_flow':
        golden_general_flow()
        sys.exit(0)
    if os.environ.get('ACB_GOLDEN_ONLY') == 'fprocess':
        golden_fprocess()
        sys.exit(0)
    if os.environ.get('ACB_GOLDEN_ONLY') == 'cleansc_custom':
        golden_cleansc_custom()
        sys.exit(0)
    if os.environ.get('ACB_GOLDEN_ONLY') == 'functional_orth_cleansc':
        golden_functional_orth_cleansc()
        sys.exit(0)
    if os.environ.get('ACB_GOLDEN_ONLY') == 'psf_damas':
        golden_psf_damas()
        sys.exit(0)
    if os.environ.get('ACB_GOLDEN_ONLY') == 'eig':
        golden_eig()
        sys.exit(0)
    if os.environ.get('ACB_GOLDEN_ONLY') == 'custom_flow':
        golden_custom_flow()
        sys.exit(0)
    golden_env()
    golden_small()
    golden_rank1()
    golden_config1()
    golden_eig()
    golden_custom_flow()
    golden_psf_damas()
    golden_functional_orth_cleansc()
    golden_cleansc_custom()
    golden_fprocess()
    golden_general_flow()
