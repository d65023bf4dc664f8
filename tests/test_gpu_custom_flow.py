"""Custom steering vectors and the uniform-flow environment on the GPU against the reference's own
results (tests/golden/custom_flow_kat.npz).  Bar: the plain form's 1e-10 of the max per bin."""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

STEERS = ['classic', 'inverse', 'true level', 'true location']
TOL = 1e-10


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_custom_steering_kernels_vs_reference(golden):
    from acoular_b200 import fastFuncs as F
    g = golden('custom_flow_kat.npz')
    s = golden('small_kat.npz')
    csm = s['csm0']
    M = s['mpos'].shape[1]
    for j, b in enumerate(g['bins']):
        for st in STEERS:
            h = np.ascontiguousarray(g[f'steer_{st.replace(" ", "_")}_{b}'])
            for rd in (False, True):
                res, nrm = F.beamformerFreq('custom', rd, 1.25, h, np.ascontiguousarray(csm[b]))
                assert _rel(res, g[f'cust_{st.replace(" ", "_")}_{int(rd)}_{b}']) <= TOL
                assert _rel(nrm, g[f'custn_{st.replace(" ", "_")}_{int(rd)}_{b}']) <= TOL
                res, _ = F.beamformerFreq('custom', rd, 1.25, h, (np.array(g['eigvals'][j, M - 2:]),
                                                                  np.ascontiguousarray(g['eigvecs'][j][:, M - 2:])))
                assert _rel(res, g[f'custe_{st.replace(" ", "_")}_{int(rd)}_{b}']) <= TOL


def test_uniform_flow_beamformer_vs_reference(golden):
    """BeamformerBase with a SteeringVector in a UniformFlowEnvironment: the flow-corrected distances
    go to the map kernel as given (acb_map_rm_f64)."""
    import acoular_b200 as ac
    from acoular_b200.environments import UniformFlowEnvironment
    g = golden('custom_flow_kat.npz')
    s = golden('small_kat.npz')
    ts = ac.TimeSamples(data=s['data'], sample_freq=float(s['fs']))
    ps = ac.PowerSpectra(source=ts, block_size=128, window='Hanning', overlap='50%')
    env = UniformFlowEnvironment(c=343.0, ma=0.3, fdv=(1.0, 0.5, 0.0))
    grid, mics = ac.ImportGrid(pos=s['gpos']), ac.MicGeom(pos_total=s['mpos'])
    for st in STEERS:
        for rd in (False, True):
            bf = ac.BeamformerBase(freq_data=ps, steer=ac.SteeringVector(grid=grid, mics=mics, steer_type=st,
                                                                         env=env), r_diag=rd)
            got = np.array(bf.result[10:31])
            ref = g[f'flow_{st.replace(" ", "_")}_{int(rd)}']
            assert float((np.abs(got - ref).max(axis=1) / np.abs(ref).max(axis=1)).max()) <= TOL, (st, rd)


def test_steering_subclass_takes_custom_path(golden):
    """A SteeringVector subclass is a custom steering object in the reference (its steer_vector is
    materialised per bin, acoular/fbeamform.py:470-472); the map equals the custom kernel's result."""
    import acoular_b200 as ac
    from acoular_b200 import fastFuncs as F
    s = golden('small_kat.npz')

    class MySteer(ac.SteeringVector):
        pass

    ts = ac.TimeSamples(data=s['data'], sample_freq=float(s['fs']))
    ps = ac.PowerSpectra(source=ts, block_size=128, window='Hanning', overlap='50%')
    st = MySteer(grid=ac.ImportGrid(pos=s['gpos']), mics=ac.MicGeom(pos_total=s['mpos']), steer_type='true level')
    bf = ac.BeamformerBase(freq_data=ps, steer=st, r_diag=True)
    got = np.array(bf.result[12])
    f = ps.fftfreq()[12]
    ref, _ = F.beamformerFreq('custom', True, bf.sig_loss_norm(), np.ascontiguousarray(st.steer_vector(f)),
                              np.ascontiguousarray(s['csm0'][12]))
    ref = np.where(ref < 0, 0.0, ref)
    assert _rel(got, ref) <= 1e-12
    # and it agrees with the predefined-type fast path to the steering restatement's float32 accuracy
    bf0 = ac.BeamformerBase(freq_data=ps, steer=ac.SteeringVector(grid=st.grid, mics=st.mics, steer_type='true level'),
                            r_diag=True)
    assert _rel(got, np.array(bf0.result[12])) <= 1e-5


def test_general_flow_environment_map(golden):
    """BeamformerBase with the ray-traced GeneralFlowEnvironment (a rotating flow): the map kernel takes
    the environment's apparent distances as given; compared with the oracle on the same distances."""
    import warnings

    import acoular_b200 as ac
    from oracle import oracle as O
    s = golden('small_kat.npz')
    env = ac.GeneralFlowEnvironment(c=343.0, ff=ac.RotatingFlow(rps=3.0, v0=2.0), N=200)   # rays cover the grid
    ts = ac.TimeSamples(data=s['data'], sample_freq=float(s['fs']))
    ps = ac.PowerSpectra(source=ts, block_size=128, window='Hanning', overlap='50%')
    st = ac.SteeringVector(grid=ac.ImportGrid(pos=s['gpos']), mics=ac.MicGeom(pos_total=s['mpos']), env=env,
                           steer_type='true level')
    with warnings.catch_warnings():
        warnings.simplefilter('ignore', RuntimeWarning)
        r0, rm = np.atleast_1d(st.r0), st.rm
    assert np.isfinite(rm).all() and np.isfinite(r0).all()
    bf = ac.BeamformerBase(freq_data=ps, steer=st, r_diag=True)
    ind = np.arange(10, 31)
    got = np.array(bf.result[10:31])
    ref = O.beamformer_calc(ps.csm, ps.fftfreq(), ind, r0, rm, 343.0, 'true level', True)[ind]
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()
