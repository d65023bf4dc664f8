"""BeamformerFunctional, BeamformerOrth and BeamformerCleansc on the GPU against the reference's own
results (tests/golden/functional_orth_cleansc_kat.npz: its _calc methods with its eigh, calcTransfer and
numba kernels) and the oracle.

Tolerances: Functional and Orth maps <= 1e-8 of max end to end (device CSM and eigh against the
reference's; the eigenvalues of these fixtures are well separated, smallest 3e-4 of the largest).
CLEAN-SC results are float32 in the reference too: the same peaks, values <= 1e-5 of max (the
iterations feed each peak's float32 phase and the maps back into the CSM; sums over mics run in
another order than numpy's BLAS calls).
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

STEERS = ['classic', 'inverse', 'true level', 'true location']


def _rel(a, b):
    return float(np.abs(np.asarray(a) - b).max() / np.abs(b).max())


@pytest.fixture(scope='module')
def cases(golden):
    import acoular_b200 as ac
    from acoular_b200 import workloads
    s = golden('small_kat.npz')
    c1 = golden('config1_band.npz')
    ts = ac.TimeSamples(data=s['data'], sample_freq=float(s['fs']))
    ps_s = ac.PowerSpectra(source=ts, block_size=128, window='Hanning', overlap='50%')
    wl = workloads.three_sources_64()
    csm = np.zeros((c1['freqs'].size, 64, 64), dtype=np.complex128)
    csm[c1['band_bins']] = c1['csm_band']
    ps_c = ac.PowerSpectraImport(csm=csm, frequencies=c1['freqs'])
    return {
        's': (ps_s, ac.MicGeom(pos_total=s['mpos']), ac.ImportGrid(pos=s['gpos']), s['csm0'], s['freqs0']),
        'c1': (ps_c, wl.mics, wl.grid, csm, c1['freqs']),
    }


def _steer(ac, mics, grid, st):
    return ac.SteeringVector(grid=grid, mics=mics, steer_type=st)


@pytest.mark.parametrize('tag', ['s', 'c1'])
def test_functional_vs_reference(golden, cases, tag):
    import acoular_b200 as ac
    g = golden('functional_orth_cleansc_kat.npz')
    ps, mics, grid, _, _ = cases[tag]
    ind = g[f'{tag}_bins']
    for st in STEERS:
        for gamma in (1.0, 3.0):
            bf = ac.BeamformerFunctional(freq_data=ps, steer=_steer(ac, mics, grid, st), gamma=gamma)
            got = np.array([bf.result[int(i)] for i in ind])
            assert _rel(got, g[f'{tag}_functional_{st.replace(" ", "_")}_g{gamma:g}']) <= 1e-8, (st, gamma)
    with pytest.raises(ValueError):
        ac.BeamformerFunctional(freq_data=ps, steer=_steer(ac, mics, grid, 'classic'), r_diag=True)


@pytest.mark.parametrize('tag', ['s', 'c1'])
def test_orth_vs_reference(golden, cases, tag):
    import acoular_b200 as ac
    g = golden('functional_orth_cleansc_kat.npz')
    ps, mics, grid, _, _ = cases[tag]
    ind = g[f'{tag}_bins']
    M = mics.num_mics
    for st in STEERS:
        for rd in (False, True):
            for el in ([-1], [-1, -2, -3], [M - 6, 2]):
                ref = g[f'{tag}_orth_{st.replace(" ", "_")}_{int(rd)}_{"_".join(str(e) for e in el)}']
                if el == [-1, -2, -3]:
                    bf = ac.BeamformerOrth(freq_data=ps, steer=_steer(ac, mics, grid, st), r_diag=rd, n=3)
                    assert list(bf.eva_list) == el
                else:
                    bf = ac.BeamformerOrth(freq_data=ps, steer=_steer(ac, mics, grid, st), r_diag=rd, eva_list=el)
                got = np.array([bf.result[int(i)] for i in ind])
                assert np.array_equal(got != 0, ref != 0), (st, rd, el)
                assert _rel(got, ref) <= 1e-8, (st, rd, el)


@pytest.mark.parametrize('tag', ['s', 'c1'])
def test_cleansc_vs_reference(golden, cases, tag):
    import acoular_b200 as ac
    g = golden('functional_orth_cleansc_kat.npz')
    ps, mics, grid, _, _ = cases[tag]
    ind = g[f'{tag}_bins']
    for st in STEERS:
        for rd in (False, True):
            for n_iter, damp, stopn in ((0, 0.6, 3), (10, 0.9, 4)):
                ref = g[f'{tag}_cleansc_{st.replace(" ", "_")}_{int(rd)}_{n_iter}_{damp:g}_{stopn}']
                bf = ac.BeamformerCleansc(freq_data=ps, steer=_steer(ac, mics, grid, st), r_diag=rd, n_iter=n_iter,
                                          damp=damp, stopn=stopn)
                got = np.array([bf.result[int(i)] for i in ind])
                assert np.array_equal(got != 0, ref != 0), (st, rd, n_iter)
                assert _rel(got, ref) <= 1e-5, (st, rd, n_iter)


def test_cleansc_kernel_flow_and_single_bins(golden):
    """The device loop on given (uniform-flow) distances, bins one at a time and all at once, against
    the oracle's restatement."""
    from acoular_b200 import device as D
    s = golden('small_kat.npz')
    f = golden('custom_flow_kat.npz')
    csm, freqs = s['csm0'], s['freqs0']
    r0, rm = f['flow_r0'], f['flow_rm']
    ind = np.array([11, 19, 27])
    M = rm.shape[1]
    for st in ('classic', 'true location'):
        for rd in (False, True):
            norm = O.sig_loss_norm(rd, M)
            ref = O.beamformer_cleansc_calc(csm, freqs, ind, r0, rm, 343.0, st, rd, 12, 0.7, 3)[ind]
            k = torch.as_tensor(2 * np.pi * freqs[ind] / 343.0, device='cuda')
            c = torch.as_tensor(csm[ind], device='cuda')
            r0d, rmd = torch.as_tensor(r0, device='cuda'), torch.as_tensor(rm, device='cuda')
            got = D.cleansc_f64(c, k, st, rd, norm, 12, 0.7, 3, r0=r0d, rm=rmd).double().cpu().numpy()
            assert np.array_equal(got != 0, ref != 0) and _rel(got, ref) <= 1e-5, (st, rd)
            one = D.cleansc_f64(c[1:2], k[1:2], st, rd, norm, 12, 0.7, 3, r0=r0d, rm=rmd).double().cpu().numpy()
            assert np.array_equal(one[0], got[1])
            assert np.array_equal(c.cpu().numpy(), csm[ind])   # the caller's CSM is left unchanged


def test_cleansc_errors(cases):
    import acoular_b200 as ac
    ps, mics, grid, _, _ = cases['s']
    with pytest.raises(ValueError):
        ac.BeamformerCleansc(freq_data=ps, steer=_steer(ac, mics, grid, 'classic'), damp=0.0)

    class MySteer(ac.SteeringVector):
        pass

    # a subclass takes the custom-steering route (its materialised steer_vector); with the plain vectors it
    # cleans the same peaks as the plain SteeringVector, within the float32 result's rounding
    got = np.asarray(ac.BeamformerCleansc(freq_data=ps, steer=MySteer(grid=grid, mics=mics)).result[20])
    ref = np.asarray(ac.BeamformerCleansc(freq_data=ps, steer=ac.SteeringVector(grid=grid, mics=mics)).result[20])
    assert np.array_equal(got != 0, ref != 0)
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()


def test_cleansc_custom_steering_object(golden):
    """BeamformerCleansc with a steering object of its own (a SteeringVector subclass whose steer_vector is
    the plain one shaded per mic) runs the custom-steering iterations (acb_cleansc_custom_f64) and gives the
    reference's result on that object (tests/golden/cleansc_custom_kat.npz): the same peaks, <= 1e-5 of max."""
    import acoular_b200 as ac
    s = golden('small_kat.npz')
    g = golden('cleansc_custom_kat.npz')
    M = s['mpos'].shape[1]
    shade = 0.5 + 0.5 * np.cos(np.pi * (np.arange(M) - (M - 1) / 2) / M)

    class ShadedSteering(ac.SteeringVector):
        def steer_vector(self, f, ind=None):
            return super().steer_vector(f, ind) * shade[np.newaxis, :]

    ps = ac.PowerSpectraImport(csm=s['csm0'], frequencies=s['freqs0'])
    ind = g['bins']
    for st in ('true level', 'classic'):
        steer = ShadedSteering(grid=ac.ImportGrid(pos=s['gpos']), mics=ac.MicGeom(pos_total=s['mpos']), steer_type=st)
        for rd in (False, True):
            for n_iter, damp, stopn in ((0, 0.6, 3), (10, 0.9, 4)):
                bf = ac.BeamformerCleansc(freq_data=ps, steer=steer, r_diag=rd, n_iter=n_iter, damp=damp, stopn=stopn)
                got = np.array([bf.result[int(i)] for i in ind])
                ref = g[f'{st.replace(" ", "_")}_{int(rd)}_{n_iter}_{damp:g}_{stopn}']
                assert np.array_equal(got != 0, ref != 0), (st, rd, n_iter)
                assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max(), (st, rd, n_iter)
