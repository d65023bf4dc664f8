"""CPU tests of the host logic of the eigen-path, deconvolution and streaming classes, and of the argument
checks of their C-ABI entry points (no GPU needed: every check below returns before any CUDA call)."""

import ctypes

import numpy as np
import pytest
from scipy import fft

import acoular_b200 as ac
from acoular_b200 import _native as N
from oracle import oracle as O


@pytest.fixture(scope='module')
def native():
    from acoular_b200 import build
    build.build()
    return N.lib()


def test_c_abi_argument_checks(native):
    p = N.MapParams()
    p.num_mics, p.num_grid, p.num_bins, p.steer_type = 8, 81, 1, 3
    # PSF: null pointers, bad steering type, empty sources
    assert native.acb_psf_f64(ctypes.byref(p), 3, None, 1.0, None, None, 0, None, None) == N.ACB_ERR_ARG
    p.steer_type = 7
    assert native.acb_psf_f64(ctypes.byref(p), 3, 1, 1.0, 1, 1, 0, 1, None) == N.ACB_ERR_ARG
    p.steer_type = 3
    assert native.acb_psf_f64(ctypes.byref(p), 0, 1, 1.0, 1, 1, 0, 1, None) == N.ACB_ERR_SHAPE
    # DAMAS: null pointers, empty grid, negative iterations
    assert native.acb_damas_gauss_seidel_f64(None, 10, 1, 1, 1, 1, 1.0, 0, None) == N.ACB_ERR_ARG
    assert native.acb_damas_gauss_seidel_f64(1, 0, 1, 1, 1, 1, 1.0, 0, None) == N.ACB_ERR_SHAPE
    assert native.acb_damas_gauss_seidel_f64(1, 10, 1, 1, 1, -1, 1.0, 0, None) == N.ACB_ERR_SHAPE
    # CLEAN-SC: workspace sizes and argument checks
    assert native.acb_cleansc_workspace_bytes(1, 81, 1, 0) == 0
    small = native.acb_cleansc_workspace_bytes(8, 81, 2, 10)
    assert small > 0
    assert native.acb_cleansc_workspace_bytes(64, 81, 2, 0) > native.acb_cleansc_workspace_bytes(64, 81, 2, 10)
    assert native.acb_cleansc_f64(ctypes.byref(p), None, 1, 1, 1, None, None, 0, 0.6, 3, 1, 1, small,
                                  None) == N.ACB_ERR_ARG
    assert native.acb_cleansc_f64(ctypes.byref(p), 1, 1, None, None, None, None, 0, 0.6, 3, 1, 1, small,
                                  None) == N.ACB_ERR_ARG                  # no geometry
    assert native.acb_cleansc_f64(ctypes.byref(p), 1, 1, 1, 1, None, None, 0, 0.6, 3, 1, 1, 16,
                                  None) == N.ACB_ERR_WORKSPACE
    # spectra generators
    assert native.acb_spectra_workspace_bytes(8, 128, 10) == 65 * 10 * 8 * 16
    assert native.acb_spectra(1, N.F64, 1000, 8, 96, 48, 0, 2, 1, 1, N.C128, 1.0, 0, 1, 1, 1 << 20,
                              None) == N.ACB_ERR_SHAPE                    # not a power of two
    assert native.acb_spectra(1, N.F64, 1000, 8, 128, 64, 0, 20, 1, 1, N.C128, 1.0, 0, 1, 1, 1 << 20,
                              None) == N.ACB_ERR_SHAPE                    # windows past the samples
    assert native.acb_spectra(1, N.F64, 1000, 8, 128, 64, 0, 2, 1, 1, N.C128, 1.0, 0, 1, 1, 16,
                              None) == N.ACB_ERR_WORKSPACE
    assert native.acb_auto_spectra(1, 0, N.C128, 0, 1.0, 1, None) == N.ACB_OK   # nothing to do
    assert native.acb_auto_spectra(1, 4, 9, 0, 1.0, 1, None) == N.ACB_ERR_ARG
    assert native.acb_cross_spectra(1, 1, 65, 8, 9, 1.0, 1, None) == N.ACB_ERR_ARG
    assert native.acb_cross_spectra(1, 0, 65, 8, N.C128, 1.0, 1, None) == N.ACB_OK


def test_rfft_and_power_spectra_settings():
    ts = ac.TimeSamples(data=np.zeros((5000, 3)), sample_freq=48000.0)
    rf = ac.RFFT(source=ts, block_size=256, window='Hanning', overlap='75%', scaling='amplitude')
    assert rf.num_freqs == 129 and rf.num_channels == 3 and rf.num_samples == 5000 // 256
    np.testing.assert_array_equal(rf.freqs, abs(fft.fftfreq(256, 1 / 48000.0)[:129]))
    with pytest.raises(ValueError, match='Block size must be even'):
        rf.block_size = 255
    for bad in ({'window': 'Kaiser'}, {'overlap': '33%'}, {'precision': 'float32'}, {'scaling': 'psd'}):
        with pytest.raises(ValueError):
            ac.RFFT(source=ts, **bad)
    w = np.hanning(256)
    assert rf._scale_value() == 1 / w.sum()
    rf.scaling = 'energy'
    assert rf._scale_value() == 1 / np.sqrt(np.dot(w, w) / 256)
    for sc in ('power', 'psd'):
        for ss in (True, False):
            aps = ac.AutoPowerSpectra(source=rf, scaling=sc, single_sided=ss)
            assert aps._get_scaling_value() == O.power_scale(256, 48000.0, sc, ss)
            assert aps.num_channels == 3 and aps.num_freqs == 129 and aps.block_size == 256
    with pytest.raises(ValueError):
        ac.AutoPowerSpectra(source=rf, precision='complex128')
    assert ac.CrossPowerSpectra(source=rf).num_channels == 9
    assert ac.CrossPowerSpectra(source=rf, calc_mode='upper').num_channels == 6
    assert ac.CrossPowerSpectra(source=rf, calc_mode='lower').num_channels == 6
    with pytest.raises(ValueError):
        ac.CrossPowerSpectra(source=rf, calc_mode='diag')
    with pytest.raises(ValueError):
        ac.CrossPowerSpectra(source=rf, precision='float64')


def _bf_parts():
    mics = ac.MicGeom(pos_total=np.random.default_rng(0).normal(size=(3, 8)))
    grid = ac.RectGrid(x_min=-0.2, x_max=0.2, y_min=-0.2, y_max=0.2, z=-0.3, increment=0.1)
    ps = ac.PowerSpectraImport(csm=np.zeros((3, 8, 8), complex), frequencies=np.array([100.0, 200.0, 300.0]))
    return ps, ac.SteeringVector(grid=grid, mics=mics)


def test_eigen_path_and_deconvolution_settings():
    ps, st = _bf_parts()
    orth = ac.BeamformerOrth(freq_data=ps, steer=st)
    assert orth.n == 1 and list(orth.eva_list) == [-1]
    orth.n = 3
    assert list(orth.eva_list) == [-1, -2, -3]
    orth.eva_list = [5, 2]
    assert list(orth.eva_list) == [5, 2]
    assert list(ac.BeamformerOrth(freq_data=ps, steer=st, n=2).eva_list) == [-1, -2]
    assert list(ac.BeamformerOrth(freq_data=ps, steer=st, n=2, eva_list=[4]).eva_list) == [4]
    fn = ac.BeamformerFunctional(freq_data=ps, steer=st, gamma=4)
    assert fn.r_diag is False and fn.r_diag_norm == 1.0 and fn.gamma == 4.0
    with pytest.raises(ValueError):
        ac.BeamformerFunctional(freq_data=ps, steer=st, r_diag=True)
    cs = ac.BeamformerCleansc(freq_data=ps, steer=st)
    assert (cs.n_iter, cs.damp, cs.stopn) == (0, 0.6, 3)
    for damp in (0.0, 1.5):
        with pytest.raises(ValueError):
            ac.BeamformerCleansc(freq_data=ps, steer=st, damp=damp)
    dm = ac.BeamformerDamas(freq_data=ps, steer=st)
    assert (dm.n_iter, dm.damp, dm.psf_precision, dm.calcmode) == (100, 1.0, 'float64', 'full')
    with pytest.raises(ValueError):
        ac.BeamformerDamas(freq_data=ps, steer=st, psf_precision='float16')
    with pytest.raises(ValueError):
        ac.BeamformerDamas(freq_data=ps, steer=st, calcmode='partial')
    psf = ac.PointSpreadFunction(steer=st, grid_indices=[1, 3])
    assert psf.calcmode == 'single' and psf.precision == 'float64' and psf.freq == 1.0
    with pytest.raises(ValueError):
        ac.PointSpreadFunction(steer=st, calcmode='lazy')
    # every digest differs by the class and its settings
    digests = {b.digest for b in (orth, fn, cs, dm, ac.BeamformerCleansc(freq_data=ps, steer=st, stopn=4),
                                  ac.BeamformerDamas(freq_data=ps, steer=st, n_iter=10))}
    assert len(digests) == 6


def test_oracle_cleansc_known_answer():
    """CLEAN-SC of the rank-1 CSM of one monopole at a grid point, classic steering (whose map of a
    monopole peaks at the source): one iteration puts float32(damp * peak) at the source and nothing
    elsewhere; more iterations keep the source as the largest entry."""
    g = O.rect_grid_pos(-0.5, 0.5, -0.5, 0.5, 1.0, 0.25)[0]
    rng = np.random.RandomState(1)
    mpos = rng.normal(size=(3, 6))
    r0, rm = O.apparent_r(g), O.apparent_r(g, mpos)
    f = 2000.0
    k = 2 * np.pi * f / 343.0
    src = 12                                   # the grid centre (0, 0, 1)
    a = O.transfer(r0[src:src + 1], rm[src:src + 1], k)[0]
    csm = np.outer(a, a.conj())[None]
    h = O.beamformer_freq('classic', False, 1.0, r0, rm, k, csm[0])[0]
    assert h.argmax() == src
    one = O.beamformer_cleansc_calc(csm, np.array([f]), [0], r0, rm, 343.0, 'classic', False, 1, 0.6, 3)[0]
    assert one[src] == np.float32(0.6 * h[src]) and np.count_nonzero(one) == 1
    more = O.beamformer_cleansc_calc(csm, np.array([f]), [0], r0, rm, 343.0, 'classic', False, 0, 0.6, 3)[0]
    assert more.argmax() == src


def test_flow_fields_and_general_flow_environment_match_reference(golden):
    """SlotJet / OpenJet / RotatingFlow velocities and Jacobians, spiral_sphere and the ray-traced
    GeneralFlowEnvironment.apparent_r against the reference's (tests/golden/general_flow_kat.npz).

    Tolerances: the fields and the ray directions are the same formulas evaluated in another order
    (<= 1e-14 of max).  The apparent distances agree to <= 5e-5 of max (measured 1.1e-5): the reference
    integrates each ray with VODE at rtol 1e-4, the batched Dormand-Prince steps here at 1e-9, so the
    sampled ray positions, and with them the piecewise-linear travel times, differ by VODE's error.
    Distances through the smooth rotating flow agree to 1e-6."""
    import warnings

    from acoular_b200.environments import spiral_sphere

    def close(a, b, tol):
        assert a.shape == b.shape
        assert np.abs(a - b).max() <= tol * np.abs(b).max(), np.abs(a - b).max() / np.abs(b).max()

    g = golden('general_flow_kat.npz')
    fields = {'openjet': ac.OpenJet(v0=20.0, D=0.4, l=6.2), 'slotjet': ac.SlotJet(v0=15.0, B=0.3, l=5.2),
              'rotating': ac.RotatingFlow(rps=2.0, v0=3.0)}
    with warnings.catch_warnings():
        warnings.simplefilter('error', RuntimeWarning)   # no division warnings leak out of the fields
        for name, ff in fields.items():
            vs, js = zip(*[ff.v(p) for p in g['pts']])
            close(np.array(vs), g[f'{name}_v'], 1e-14)
            close(np.array(js), g[f'{name}_jac'], 1e-14)
            vel, jac = ff.field(g['pts'].T)          # the batched form gives the same values
            close(vel.T, g[f'{name}_v'], 1e-14)
            close(np.moveaxis(jac, 2, 0), g[f'{name}_jac'], 1e-14)
            env = ac.GeneralFlowEnvironment(c=343.0, ff=ff, N=64, Om=np.pi)
            tol = 1e-6 if name == 'rotating' else 5e-5
            close(env.apparent_r(g['gpos'], g['mpos']), g[f'{name}_rm'], tol)
            close(env.apparent_r(g['gpos']), g[f'{name}_r0'], tol)
            assert len(env.idict) == 4          # one travel-time field per position (3 mics, the origin), reused
    close(spiral_sphere(40, np.pi, b=np.array((0.3, -0.5, 1.0))), g['sphere'], 1e-14)


def test_general_flow_uniform_field_matches_closed_form():
    """A constant flow field traced by GeneralFlowEnvironment against UniformFlowEnvironment's closed form
    (acoular/environments.py:290-332): rays are straight, so what remains is the piecewise-linear
    interpolation of the travel times between ray samples (measured 1.6e-3 of the distance at N = 400, 7.4e-3 at
    N = 100; the flow itself changes the distances by 8 %)."""
    from acoular_b200.environments import FlowField

    class Constant(FlowField):
        def __init__(self, vel):
            self.vel = np.asarray(vel, dtype=np.float64)

        def field(self, x):
            n = np.asarray(x).shape[1]
            return np.repeat(self.vel[:, None], n, axis=1), np.zeros((3, 3, n))

    ma = 0.15
    gpos = np.stack(np.meshgrid(np.linspace(-0.2, 0.2, 5), np.linspace(-0.2, 0.2, 5), [0.7], indexing='ij')).reshape(3, -1)
    mpos = np.array(((0.1, -0.3, 0.0), (-0.2, 0.05, 0.02))).T
    ray = ac.GeneralFlowEnvironment(c=343.0, ff=Constant((ma * 343.0, 0.0, 0.0)), N=400, Om=np.pi)
    exact = ac.UniformFlowEnvironment(c=343.0, ma=ma, fdv=(1.0, 0.0, 0.0))
    got, ref = ray.apparent_r(gpos, mpos), exact.apparent_r(gpos, mpos)
    assert np.isfinite(got).all()
    assert np.abs(got - ref).max() <= 3e-3 * ref.max()


def test_heevd_select_argument_checks(native):
    """acb_heevd_select_f64 rejects bad requests before any CUDA call: null pointers (ACB_ERR_ARG), rank counts
    outside 1..4 or above M (ACB_ERR_SHAPE), ranks outside 0..M-1 (ACB_ERR_ARG), sizes whose work arrays exceed
    the shared memory (ACB_ERR_UNSUPPORTED) and a short workspace (ACB_ERR_WORKSPACE)."""
    sel = (ctypes.c_int * 4)(0, 1, 2, 3)
    ws = native.acb_heevd_workspace_bytes(8, 2)
    call = native.acb_heevd_select_f64
    assert call(None, 2, 8, 1, sel, 1, 1, 1, ws, None) == N.ACB_ERR_ARG
    assert call(1, 2, 8, 1, None, 1, 1, 1, ws, None) == N.ACB_ERR_ARG
    assert call(1, 2, 8, 0, sel, 1, 1, 1, ws, None) == N.ACB_ERR_SHAPE
    assert call(1, 2, 8, 5, sel, 1, 1, 1, ws, None) == N.ACB_ERR_SHAPE
    assert call(1, 2, 3, 4, sel, 1, 1, 1, ws, None) == N.ACB_ERR_SHAPE        # more ranks than mics
    bad = (ctypes.c_int * 1)(8)
    assert call(1, 2, 8, 1, bad, 1, 1, 1, ws, None) == N.ACB_ERR_ARG           # rank M
    assert call(1, 1, 4000, 1, sel, 1, 1, 1, 1 << 40, None) == N.ACB_ERR_UNSUPPORTED
    assert call(1, 2, 8, 1, sel, 1, 1, 1, ws - 1, None) == N.ACB_ERR_WORKSPACE
