"""The CPU oracle against golden vectors produced by running the reference's own code.

The oracle (``oracle/``) restates the reference's numba kernels in C and its glue in numpy; these
tests pin it bit-for-bit (or to the stated tolerance) before it is trusted as the GPU checker.
"""

import numpy as np
import pytest

from oracle import oracle as O

STEERS = ['classic', 'inverse', 'true level', 'true location']


def test_apparent_r_matches_reference_regression(golden):
    d = golden('env_apparent_r.npz')
    res_arr = np.vstack((O.apparent_r(d['gpos'], d['mpos']).T, O.apparent_r(d['gpos']).T))
    res_sc = np.vstack((O.apparent_r(d['gpos'], 0.0).T, O.apparent_r(d['gpos']).T))
    # the reference's own snapshot tolerance (tests/regression/test_environments.py:66)
    np.testing.assert_allclose(res_arr, d['mics_arr'], rtol=1e-5, atol=1e-8)
    np.testing.assert_allclose(res_sc, d['mics_scalar'], rtol=1e-5, atol=1e-8)
    assert np.array_equal(O.apparent_r(d['gpos'], d['mpos']), d['rm_ref'])


@pytest.mark.parametrize('case', range(5))
def test_calc_csm_bit_exact(golden, case):
    d = golden('small_kat.npz')
    bs, win, ov, prec = d[f'csm{case}_case']
    csm = O.calc_csm(d['data'], int(bs), str(win), str(ov), str(prec))
    ref = d[f'csm{case}']
    assert csm.dtype == ref.dtype
    assert np.array_equal(csm, ref)
    np.testing.assert_array_equal(O.fftfreq(int(bs), float(d['fs'])), d[f'freqs{case}'])


def test_num_blocks_formula():
    # 2000 samples, block 128, 50 %: the formula gives 30.25 while 30 windows exist
    assert O.num_blocks(2000, 128, 2) == 30.25
    assert sum(1 for _ in O.source_windows(np.zeros((2000, 2)), 128, 2)) == 30
    assert O.num_blocks(51200, 128, 2) == 799


@pytest.mark.parametrize('steer', STEERS)
@pytest.mark.parametrize('r_diag', [False, True])
def test_beamformer_bit_exact(golden, steer, r_diag):
    d = golden('small_kat.npz')
    r0 = O.apparent_r(d['gpos'])
    rm = O.apparent_r(d['gpos'], d['mpos'])
    res = O.beamformer_calc(d['csm0'], d['freqs0'], d['bins'], r0, rm, 343.0, steer, r_diag)
    key = f'map_{steer.replace(" ", "_")}_{int(r_diag)}'
    assert np.array_equal(res[d['bins']], d[key])
    syn = O.synthetic(res, d['freqs0'], 8000.0, 3, tuple(d['gshape']))
    np.testing.assert_allclose(syn, d['syn_' + key], rtol=1e-14, atol=0)


def test_reference_position_and_rdiag_norm(golden):
    d = golden('small_kat.npz')
    ref = np.array([0.1, -0.05, 0.02])
    r0 = O.apparent_r(d['gpos'], ref[:, None])
    np.testing.assert_array_equal(r0, d['r0_ref'])
    rm = O.apparent_r(d['gpos'], d['mpos'])
    res = O.beamformer_calc(d['csm0'], d['freqs0'], d['bins'], r0, rm, 343.0, 'true level', True, r_diag_norm=1.25)
    assert np.array_equal(res[d['bins']], d['map_ref_rdn'])


@pytest.mark.parametrize('steer', STEERS)
@pytest.mark.parametrize('r_diag', [False, True])
def test_rank1_known_answer(golden, steer, r_diag):
    d = golden('rank1_kat.npz')
    r0 = O.apparent_r(d['gpos'])
    rm = O.apparent_r(d['gpos'], d['mpos'])
    res = O.beamformer_calc(d['csm'], d['freqs'], [0], r0, rm, 343.0, steer, r_diag)
    assert np.array_equal(res[0], d[f'map_{steer.replace(" ", "_")}_{int(r_diag)}'])
    if steer == 'true level' and not r_diag:
        # true-level steering recovers the source level at the source position (0, 0, 1)
        g = int(np.argmin(np.sum((d['gpos'] - np.array([[0], [0], [1.0]])) ** 2, 0)))
        assert abs(res[0, g] - 1.0) < 1e-6


def test_config1_band_goldens(golden):
    """The 64-mic three-source workload: restated time data, CSM band and all 8 maps."""
    from acoular_b200 import workloads
    d = golden('config1_band.npz')
    wl = workloads.three_sources_64()
    data = wl.time_data()
    np.testing.assert_allclose([data.sum(), (data ** 2).sum(), data[::997, ::7].sum()], d['data_stats'], rtol=1e-12)
    csm = O.calc_csm(data, 128, 'Hanning', '50%', 'complex128')
    scale = np.abs(d['csm_band']).max()
    assert np.abs(csm[18:23] - d['csm_band']).max() <= 1e-12 * scale
    g = wl.grid
    r0 = O.apparent_r(g.pos)
    rm = O.apparent_r(g.pos, wl.mics.pos)
    for steer in STEERS:
        for r_diag in (False, True):
            # only the band bins 18..22 are stored; pad the CSM so bin indices keep their wave numbers
            res = O.beamformer_calc(np.concatenate([np.zeros((18, 64, 64), complex), d['csm_band']]), d['freqs'],
                                    range(18, 23), r0, rm, 343.0, steer, r_diag)
            key = f'map_{steer.replace(" ", "_")}_{int(r_diag)}'
            assert np.array_equal(res[18:23], d[key])


# ---------------------------------------------------------------------------------------------
# eigenvalue beamformers (BeamformerEig, BeamformerMusic) against the reference's own results
# ---------------------------------------------------------------------------------------------
@pytest.mark.parametrize('tag', ['s', 'c1'])
def test_oracle_eig_beamformers_match_reference(golden, tag):
    g = golden('eig_kat.npz')
    mpos, gpos, bins, freqs = g[f'{tag}_mpos'], g[f'{tag}_gpos'], g[f'{tag}_bins'], g[f'{tag}_freqs']
    eva, eve = g[f'{tag}_eigvals'], g[f'{tag}_eigvecs']
    r0, rm = O.apparent_r(gpos), O.apparent_r(gpos, mpos)
    M = mpos.shape[1]
    ind = np.arange(len(bins))
    for n in (-1, 0, M // 2):
        assert int(g[f'{tag}_eig_n{n}_na']) == O.eig_na(n, M)
        for st in STEERS:
            for rd in (False, True):
                ref = g[f'{tag}_eig_n{n}_{st.replace(" ", "_")}_{int(rd)}']
                got = O.beamformer_eig_calc(eva, eve, freqs, ind, r0, rm, 343.0, st, rd, n=n)
                np.testing.assert_array_equal(got, ref)
    for n in (1, 3):
        for st in STEERS:
            ref = g[f'{tag}_music_n{n}_{st.replace(" ", "_")}']
            got = O.beamformer_music_calc(eva, eve, freqs, ind, r0, rm, 343.0, st, n=n)
            np.testing.assert_allclose(got, ref, rtol=1e-13, atol=0)


# ---------------------------------------------------------------------------------------------
# custom steering vectors and the uniform-flow environment against the reference's own results
# ---------------------------------------------------------------------------------------------
def test_oracle_custom_steering_and_flow_match_reference(golden):
    g = golden('custom_flow_kat.npz')
    s = golden('small_kat.npz')
    csm, freqs, mpos, gpos = s['csm0'], s['freqs0'], s['mpos'], s['gpos']
    M = mpos.shape[1]
    for j, b in enumerate(g['bins']):
        for st in STEERS:
            h = g[f'steer_{st.replace(" ", "_")}_{b}']
            for rd in (False, True):
                ref = g[f'cust_{st.replace(" ", "_")}_{int(rd)}_{b}']
                res, nrm = O.beamformer_freq_custom(rd, 1.25, h, csm=csm[b])
                np.testing.assert_allclose(res, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
                np.testing.assert_allclose(nrm, g[f'custn_{st.replace(" ", "_")}_{int(rd)}_{b}'], rtol=1e-13)
                ref = g[f'custe_{st.replace(" ", "_")}_{int(rd)}_{b}']
                res, _ = O.beamformer_freq_custom(rd, 1.25, h, eig=(g['eigvals'][j, M - 2:],
                                                                    g['eigvecs'][j][:, M - 2:]))
                np.testing.assert_allclose(res, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    r0f = O.uniform_flow_apparent_r(gpos, 0.0, 0.3, (1.0, 0.5, 0.0))
    rmf = O.uniform_flow_apparent_r(gpos, mpos, 0.3, (1.0, 0.5, 0.0))
    np.testing.assert_array_equal(r0f, g['flow_r0'])
    np.testing.assert_array_equal(rmf, g['flow_rm'])
    ind = np.arange(10, 31)
    for st in STEERS:
        for rd in (False, True):
            got = O.beamformer_calc(csm, freqs, ind, r0f, rmf, 343.0, st, rd)[ind]
            ref = g[f'flow_{st.replace(" ", "_")}_{int(rd)}']
            if st in ('classic', 'inverse'):
                np.testing.assert_array_equal(got, ref)
            else:
                # the 1/r steering types differ from numba's complex-by-real division by 1 ulp on some
                # non-Euclidean distances (bit-exact for the Euclidean ones of small_kat.npz)
                np.testing.assert_allclose(got, ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())


def test_host_uniform_flow_and_steer_vector_match_reference(golden):
    """The package's host-side UniformFlowEnvironment and SteeringVector.steer_vector restatements."""
    import acoular_b200 as ac
    from acoular_b200.environments import UniformFlowEnvironment
    g = golden('custom_flow_kat.npz')
    s = golden('small_kat.npz')
    env = UniformFlowEnvironment(c=343.0, ma=0.3, fdv=(1.0, 0.5, 0.0))
    np.testing.assert_array_equal(env.apparent_r(s['gpos'], s['mpos']), g['flow_rm'])
    np.testing.assert_array_equal(env.apparent_r(s['gpos']), g['flow_r0'])
    st = ac.SteeringVector(grid=ac.ImportGrid(pos=s['gpos']), mics=ac.MicGeom(pos_total=s['mpos']))
    for b in g['bins']:
        for t in STEERS:
            st.steer_type = t
            ref = g[f'steer_{t.replace(" ", "_")}_{b}']
            got = st.steer_vector(s['freqs0'][b])
            # float32 cos/sin of numpy vs the reference's numba (libm): a few float32 ulp
            assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max()


def test_oracle_psf_and_damas_match_reference(golden):
    """The oracle's calcPointSpreadFunction and Gauss-Seidel restatements against the reference's
    PointSpreadFunction._psf_call and BeamformerDamas._calc (tests/golden/psf_damas_kat.npz)."""
    g = golden('psf_damas_kat.npz')
    s = golden('small_kat.npz')
    csm, freqs, mpos, gpos = s['csm0'], s['freqs0'], s['mpos'], s['gpos']
    r0, rm = O.apparent_r(gpos), O.apparent_r(gpos, mpos)
    G = gpos.shape[1]
    k = 2 * np.pi * freqs[int(g['psf_bin'])] / 343.0
    bins = g['bins']
    for st in STEERS:
        key = st.replace(' ', '_')
        np.testing.assert_allclose(O.psf(st, r0, rm, k, np.arange(G)), g[f'psf_full_{key}'], rtol=1e-14,
                                   atol=1e-14 * np.abs(g[f'psf_full_{key}']).max())
        np.testing.assert_array_equal(O.psf(st, r0, rm, k, np.arange(G), 'float32'), g[f'psf_full32_{key}'])
        np.testing.assert_array_equal(O.psf(st, r0, rm, k, g['src'], 'float32'), g[f'psf_src_{key}'])
        ref = g[f'psf_flow_{key}']
        np.testing.assert_allclose(O.psf(st, g['flow_r0'], g['flow_rm'], k, g['src']), ref, rtol=1e-14,
                                   atol=1e-14 * np.abs(ref).max())
        for rd in (False, True):
            ref = g[f'damas_{key}_{int(rd)}']
            got = O.beamformer_damas_calc(csm, freqs, bins, r0, rm, 343.0, st, rd, 10, 0.98)[bins]
            np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-13 * np.abs(ref).max())
    ref = g['damas_default_classic_0']
    got = O.beamformer_damas_calc(csm, freqs, bins, r0, rm, 343.0, 'classic', False)[bins]
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-13 * np.abs(ref).max())
    ref = g['damas_f32_true_level_1']
    got = O.beamformer_damas_calc(csm, freqs, bins, r0, rm, 343.0, 'true level', True, 10, 0.98, 'float32')[bins]
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-13 * np.abs(ref).max())


def test_oracle_gauss_seidel_known_answers():
    """Hand-checkable Gauss-Seidel cases: identity PSF returns the (clipped) map after one sweep; a
    2x2 system with relaxation follows the sweep formula row by row."""
    y = np.array([1.0, -2.0, 3.0])
    x = O.damas_gauss_seidel(np.eye(3), y, 1, 1.0, y.copy())
    np.testing.assert_array_equal(x, [1.0, 0.0, 3.0])
    A = np.array([[1.0, 0.5], [0.25, 1.0]])
    y = np.array([2.0, 1.0])
    x = O.damas_gauss_seidel(A, y, 1, 0.5, np.array([1.0, 1.0]))
    x0 = 0.5 * 1.0 + 0.5 * (2.0 - 0.5 * 1.0)
    x1 = 0.5 * 1.0 + 0.5 * (1.0 - 0.25 * x0)
    np.testing.assert_allclose(x, [x0, x1], rtol=0, atol=1e-15)


@pytest.mark.parametrize('tag', ['s', 'c1'])
def test_oracle_functional_orth_cleansc_match_reference(golden, tag):
    """The oracle's BeamformerFunctional / BeamformerOrth / BeamformerCleansc restatements against the
    reference's _calc methods (tests/golden/functional_orth_cleansc_kat.npz): bit for bit."""
    from acoular_b200 import workloads
    g = golden('functional_orth_cleansc_kat.npz')
    if tag == 's':
        s = golden('small_kat.npz')
        csm, freqs, mpos, gpos = s['csm0'], s['freqs0'], s['mpos'], s['gpos']
    else:
        c1 = golden('config1_band.npz')
        wl = workloads.three_sources_64()
        freqs, mpos, gpos = c1['freqs'], wl.mics.pos, wl.grid.pos
        csm = np.zeros((freqs.size, 64, 64), dtype=np.complex128)
        csm[c1['band_bins']] = c1['csm_band']
    ind = g[f'{tag}_bins']
    M = mpos.shape[1]
    r0, rm = O.apparent_r(gpos), O.apparent_r(gpos, mpos)
    eva, eve = np.linalg.eigh(csm)
    for st in STEERS:
        key = st.replace(' ', '_')
        for gamma in (1.0, 3.0):
            got = O.beamformer_functional_calc(eva, eve, freqs, ind, r0, rm, 343.0, st, gamma)[ind]
            np.testing.assert_array_equal(got, g[f'{tag}_functional_{key}_g{gamma:g}'])
        for rd in (False, True):
            for el in ([-1], [-1, -2, -3], [M - 6, 2]):
                got = O.beamformer_orth_calc(eva, eve, freqs, ind, r0, rm, 343.0, st, rd, el)[ind]
                np.testing.assert_array_equal(got, g[f'{tag}_orth_{key}_{int(rd)}_{"_".join(str(e) for e in el)}'])
            for n_iter, damp, stopn in ((0, 0.6, 3), (10, 0.9, 4)):
                got = O.beamformer_cleansc_calc(csm, freqs, ind, r0, rm, 343.0, st, rd, n_iter, damp, stopn)[ind]
                np.testing.assert_array_equal(got, g[f'{tag}_cleansc_{key}_{int(rd)}_{n_iter}_{damp:g}_{stopn}'])


def test_oracle_fprocess_generators_match_reference(golden):
    """The oracle's RFFT / AutoPowerSpectra / CrossPowerSpectra restatements against the reference's
    generators (tests/golden/fprocess_kat.npz): block sizes and values bit for bit."""
    g = golden('fprocess_kat.npz')
    s = golden('small_kat.npz')
    data, fs = s['data'], float(s['fs'])
    for ci in range(4):
        bs, win, ov, prec, scaling, num = g[f'rfft{ci}_case']
        bs, num = int(bs), int(num)
        blocks = list(O.rfft_blocks(data, bs, win, ov, prec, scaling, num))
        assert [b.shape[0] for b in blocks] == list(g[f'rfft{ci}_sizes'])
        np.testing.assert_array_equal(np.concatenate(blocks), g[f'rfft{ci}'])
        for ai, (sc, ss, ap) in enumerate([('power', True, 'float64'), ('psd', False, 'float32')]):
            a = np.concatenate(list(O.auto_power_blocks(blocks, O.power_scale(bs, fs, sc, ss), ap)))
            np.testing.assert_array_equal(a, g[f'aps{ci}_{ai}'])
        cprec = 'complex64' if prec == 'complex64' else 'complex128'
        scale = O.power_scale(bs, fs, 'psd' if ci % 2 else 'power', True)
        c = np.concatenate(list(O.cross_power_blocks(blocks, bs // 2 + 1, data.shape[1], scale, cprec)))
        np.testing.assert_array_equal(c[:2 * num], g[f'cps{ci}'])
        np.testing.assert_array_equal(c.astype(np.complex128).sum(axis=0), g[f'cps{ci}_sum'])


def test_oracle_cleansc_custom_steering_matches_reference(golden):
    """The oracle's CLEAN-SC with a steering object of its own (the reference's steer_vector shaded per mic;
    BeamformerCleansc routes it as 'custom', acoular/fbeamform.py:470-472, 1424-1490) against the
    reference's _calc run on the same object (tests/golden/cleansc_custom_kat.npz): the same cleaned peaks,
    values within 1e-6 of max (measured 8e-8, one float32 step of the float32 result)."""
    import acoular_b200 as ac
    s = golden('small_kat.npz')
    g = golden('cleansc_custom_kat.npz')
    M = s['mpos'].shape[1]
    shade = 0.5 + 0.5 * np.cos(np.pi * (np.arange(M) - (M - 1) / 2) / M)
    for st in ('true level', 'classic'):
        sv = ac.SteeringVector(grid=ac.ImportGrid(pos=s['gpos']), mics=ac.MicGeom(pos_total=s['mpos']), steer_type=st)
        for rd in (False, True):
            for n_iter, damp, stopn in ((0, 0.6, 3), (10, 0.9, 4)):
                got = O.beamformer_cleansc_custom_calc(s['csm0'], s['freqs0'], g['bins'],
                                                       lambda f, sv=sv: sv.steer_vector(f) * shade[None, :], rd,
                                                       n_iter, damp, stopn)[g['bins']]
                ref = g[f'{st.replace(" ", "_")}_{int(rd)}_{n_iter}_{damp:g}_{stopn}']
                assert np.array_equal(got != 0, ref != 0)
                assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max()
