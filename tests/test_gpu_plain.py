"""GPU parity of the plain FP64 path against the oracle and the reference goldens.

Tolerances (relative to the maximum magnitude of the reference array):
* CSM complex128: 1e-12 (FP64 FFT of a different radix order; identical Welch accumulation order)
* CSM complex64: 1e-5 (spectra rounded to complex64 from FP64 FFTs that differ in the last bits)
* map, glibc-faithful plain form: 1e-10 (same float32 phases and float32 cos/sin as the reference)
* map, correctly rounded float32 cos/sin (glibc_faithful=False): 1e-7
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

STEERS = ['classic', 'inverse', 'true level', 'true location']


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


@pytest.fixture(scope='module')
def dev():
    from acoular_b200 import device as D
    return D.require_cuda()


@pytest.mark.parametrize('case', range(5))
def test_csm_vs_reference_golden(golden, dev, case):
    from acoular_b200 import device as D
    d = golden('small_kat.npz')
    bs, win, ov, prec = (str(x) for x in d[f'csm{case}_case'])
    x = torch.as_tensor(d['data'], device=dev)
    csm = D.calc_csm(x, int(bs), win, ov, prec).cpu().numpy()
    ref = d[f'csm{case}']
    assert csm.dtype == ref.dtype == np.complex128
    tol = 1e-12 if prec == 'complex128' else 1e-5
    assert rel(csm, ref) <= tol
    # Hermitian structure exactly off the diagonal; the diagonal keeps the tiny imaginary residue of
    # the fused accumulation, exactly as the reference's does
    M = csm.shape[1]
    off = ~np.eye(M, dtype=bool)
    assert np.array_equal(csm[:, off], np.conj(csm.transpose(0, 2, 1))[:, off])
    diag_tol = 1e-15 if prec == 'complex128' else 1e-6
    assert np.abs(np.imag(np.einsum('fmm->fm', csm))).max() <= diag_tol * np.abs(csm).max()


def test_csm_float32_samples_and_bin_subset(dev):
    from acoular_b200 import device as D
    rng = np.random.RandomState(5)
    data = rng.randn(3000, 13).astype(np.float32)
    ref = O.calc_csm(data.astype(np.float64), 256, 'Hanning', '75%', 'complex128')
    x = torch.as_tensor(data, device=dev)
    full = D.calc_csm(x, 256, 'Hanning', '75%').cpu().numpy()
    assert rel(full, ref) <= 1e-12
    sub = D.calc_csm(x, 256, 'Hanning', '75%', bin_lo=40, num_bins=17).cpu().numpy()
    assert rel(sub, ref[40:57]) <= 1e-12
    # chunked accumulation (tiny workspace) gives the identical result
    ch = D.calc_csm(x, 256, 'Hanning', '75%', max_workspace_bytes=13 * 129 * 16 * 5).cpu().numpy()
    assert np.array_equal(ch, full)


@pytest.mark.parametrize('M,N,ov', [(1, 128, 'None'), (2, 16, '50%'), (65, 512, '87.5%'), (130, 2048, '50%'),
                                    (7, 16384, 'None'), (3, 32768, '50%'), (33, 65536, '75%')])
def test_csm_shapes(dev, M, N, ov):
    from acoular_b200 import device as D
    rng = np.random.RandomState(M + N)
    S = 2 * N + N // 3
    data = rng.randn(S, M)
    ref = O.calc_csm(data, N, 'Blackman', ov, 'complex128')
    got = D.calc_csm(torch.as_tensor(data, device=dev), N, 'Blackman', ov).cpu().numpy()
    assert rel(got, ref) <= 1e-12


def test_csm_large_blocks_all_forms(dev):
    """Blocks of 32768 and 65536 samples (sub-transforms of 8192 points and a combining pass) in every CSM
    form and a bin subset: complex128 against the oracle at 1e-12, complex64 at 1e-5, the tensor-core
    Grams within their bars of the complex128 CSM."""
    from acoular_b200 import device as D
    for N, M in ((32768, 5), (65536, 40)):
        rng = np.random.RandomState(N + M)
        data = rng.randn(3 * N, M).astype(np.float32)
        ref = O.calc_csm(data.astype(np.float64), N, 'Hanning', '50%', 'complex128')
        x = torch.as_tensor(data, device=dev)
        lo, nb = N // 8, 300
        got = D.calc_csm(x, N, 'Hanning', '50%', 'complex128', bin_lo=lo, num_bins=nb).cpu().numpy()
        assert rel(got, ref[lo:lo + nb]) <= 1e-12
        got64 = D.calc_csm(x, N, 'Hanning', '50%', 'complex64', bin_lo=lo, num_bins=nb).cpu().numpy()
        assert rel(got64, ref[lo:lo + nb]) <= 1e-5
        for prec, tol in (('tc_tf32', 2e-3), ('tc_bf16x3', 1e-4)):
            up, K = D.csm_upper_accumulate(x, N, 'Hanning', '50%', precision=prec, bin_lo=lo, num_bins=nb)
            _, w = D.window_vector('Hanning', N, dev)
            full = D.csm_finalize(up, 2.0 / N / w / D.num_blocks(3 * N, N, 2)).cpu().numpy()
            assert rel(full, ref[lo:lo + nb]) <= tol, prec


def test_csm_config1_band(golden, dev):
    from acoular_b200 import device as D, workloads
    d = golden('config1_band.npz')
    wl = workloads.three_sources_64()
    x = torch.as_tensor(wl.time_data(), device=dev)
    csm = D.calc_csm(x, 128, 'Hanning', '50%').cpu().numpy()
    assert rel(csm[18:23], d['csm_band']) <= 1e-12
    assert rel(np.real(np.einsum('fmm->fm', csm)), d['csm_diag']) <= 1e-12


def _map(dev, csm, freqs, bins, mpos, gpos, steer, r_diag, faithful=True, ref=None, rdn=0.0):
    from acoular_b200 import device as D
    M = mpos.shape[1]
    norm = O.sig_loss_norm(r_diag, M, rdn)
    c = torch.as_tensor(np.ascontiguousarray(csm[bins]), device=dev)
    k = torch.as_tensor(2 * np.pi * freqs[bins] / 343.0, device=dev)
    out = D.map_f64(c, k, torch.as_tensor(mpos, device=dev), torch.as_tensor(np.ascontiguousarray(gpos), device=dev),
                    steer, r_diag, norm, ref=ref, clip_negative=r_diag, glibc_faithful=faithful)
    return out.cpu().numpy()


@pytest.mark.parametrize('steer', STEERS)
@pytest.mark.parametrize('r_diag', [False, True])
def test_map_small_golden(golden, dev, steer, r_diag):
    d = golden('small_kat.npz')
    got = _map(dev, d['csm0'], d['freqs0'], d['bins'], d['mpos'], d['gpos'], steer, r_diag)
    ref = d[f'map_{steer.replace(" ", "_")}_{int(r_diag)}']
    assert rel(got, ref) <= 1e-10
    got_cr = _map(dev, d['csm0'], d['freqs0'], d['bins'], d['mpos'], d['gpos'], steer, r_diag, faithful=False)
    assert rel(got_cr, ref) <= 1e-7


@pytest.mark.parametrize('steer', STEERS)
@pytest.mark.parametrize('r_diag', [False, True])
def test_map_config1_golden(golden, dev, steer, r_diag):
    from acoular_b200 import workloads
    d = golden('config1_band.npz')
    wl = workloads.three_sources_64()
    csm = np.concatenate([np.zeros((18, 64, 64), complex), d['csm_band']])
    got = _map(dev, csm, d['freqs'], np.arange(18, 23), wl.mics.pos, wl.grid.pos, steer, r_diag)
    key = f'map_{steer.replace(" ", "_")}_{int(r_diag)}'
    assert rel(got, d[key]) <= 1e-10
    syn = got.sum(0).reshape(wl.grid.shape)
    assert rel(syn, d['syn_' + key]) <= 1e-10


def test_map_reference_position_and_norm(golden, dev):
    d = golden('small_kat.npz')
    got = _map(dev, d['csm0'], d['freqs0'], d['bins'], d['mpos'], d['gpos'], 'true level', True,
               ref=np.array([0.1, -0.05, 0.02]), rdn=1.25)
    assert rel(got, d['map_ref_rdn']) <= 1e-10


@pytest.mark.parametrize('steer', STEERS)
def test_map_rank1_known_answer(golden, dev, steer):
    d = golden('rank1_kat.npz')
    for r_diag in (False, True):
        got = _map(dev, d['csm'], d['freqs'], np.array([0]), d['mpos'], d['gpos'], steer, r_diag)
        assert rel(got[0], d[f'map_{steer.replace(" ", "_")}_{int(r_diag)}']) <= 1e-10


@pytest.mark.parametrize('M,G', [(2, 1), (3, 7), (5, 33), (33, 100), (130, 65), (300, 40), (513, 35)])
@pytest.mark.parametrize('steer', ['classic', 'true level'])
def test_map_shapes_vs_oracle(dev, M, G, steer):
    """Odd mic counts (row-block remainders), single/odd grid tiles, the chunked path (M > 256)."""
    rng = np.random.RandomState(M * 7 + G)
    mpos = np.vstack([rng.uniform(-0.5, 0.5, (2, M)), np.zeros((1, M))])
    gpos = np.vstack([rng.uniform(-0.4, 0.4, (2, G)), np.full((1, G), -0.6)])
    X = rng.randn(3, 2 * M, M) + 1j * rng.randn(3, 2 * M, M)
    csm = np.einsum('fkm,fkn->fmn', X.conj(), X) / (2 * M)
    freqs = np.array([1500.0, 4000.0, 9100.0])
    r0 = O.apparent_r(gpos)
    rm = O.apparent_r(gpos, mpos)
    for r_diag in (False, True):
        ref = O.beamformer_calc(csm, freqs, range(3), r0, rm, 343.0, steer, r_diag)
        got = _map(dev, csm, freqs, np.arange(3), mpos, gpos, steer, r_diag)
        assert rel(got, ref) <= 1e-10


def test_calccsm_dropin(dev):
    from acoular_b200 import fastFuncs
    rng = np.random.RandomState(11)
    for dt in (np.complex128, np.complex64):
        spec = (rng.randn(9, 70) + 1j * rng.randn(9, 70)).astype(dt)
        c0 = (rng.randn(9, 70, 70) + 1j * rng.randn(9, 70, 70)).astype(dt)
        ref = c0.copy()
        if dt == np.complex128:
            O.lib().orc_calc_csm_c128(O._dp(ref), O._dp(spec), 9, 70)
        else:
            O.lib().orc_calc_csm_c64(O._fp(ref), O._fp(spec), 9, 70)
        got = fastFuncs.calcCSM(c0.copy(), spec)
        iu = np.triu_indices(70)
        # same two-FMA accumulation as the reference: bit-identical upper triangle
        assert np.array_equal(got[:, iu[0], iu[1]], ref[:, iu[0], iu[1]])
    with pytest.raises(TypeError):
        fastFuncs.calcCSM(np.zeros((2, 3, 3)), np.zeros((2, 3)))


def test_beamformerfreq_dropin(golden, dev):
    from acoular_b200 import fastFuncs
    d = golden('small_kat.npz')
    r0 = O.apparent_r(d['gpos'])
    rm = O.apparent_r(d['gpos'], d['mpos'])
    k = 2 * np.pi * d['freqs0'][20] / 343.0
    csm = np.ascontiguousarray(d['csm0'][20])
    for steer in STEERS:
        for r_diag in (False, True):
            ref = O.beamformer_freq(steer, r_diag, 1.1, r0, rm, k, csm)
            got = fastFuncs.beamformerFreq(steer, r_diag, 1.1, (r0, rm, k), csm)
            assert rel(got[0], ref[0]) <= 1e-10
            assert rel(got[1], ref[1]) <= 1e-12
    # custom steering vectors of the wrong shape are rejected like the reference's guvectorize signature
    with pytest.raises(ValueError):
        fastFuncs.beamformerFreq('custom', True, 1.0, np.zeros((3, 8), complex), csm[:4, :4].copy())


def test_beamformer_base_end_to_end(golden, dev):
    """The public API on the 64-mic three-source workload: PowerSpectra -> BeamformerBase.synthetic."""
    import acoular_b200 as ac
    from acoular_b200 import workloads
    d = golden('config1_band.npz')
    wl = workloads.three_sources_64()
    ts = ac.TimeSamples(data=wl.time_data(), sample_freq=wl.fs)
    ps = ac.PowerSpectra(source=ts, block_size=128, window='Hanning', overlap='50%')
    for steer in STEERS:
        for r_diag in (False, True):
            st = ac.SteeringVector(grid=wl.grid, mics=wl.mics, steer_type=steer)
            bb = ac.BeamformerBase(freq_data=ps, steer=st, r_diag=r_diag)
            pm = bb.synthetic(8000, 3)
            key = 'syn_map_' + steer.replace(' ', '_') + f'_{int(r_diag)}'
            assert pm.shape == (41, 41)
            assert rel(pm, d[key]) <= 1e-10
            assert (bb._fr[18:23] == 1).all() and bb._fr.sum() == 5
    lp = ac.L_p(pm)
    assert np.isfinite(lp).all()


def test_powerspectra_streamed_upload_same_csm():
    """Pinned host samples are uploaded in chunks that overlap the CSM accumulation; the result equals
    the one-pass CSM of the same samples on the device (FP64: the same sums in the same order)."""
    import acoular_b200 as ac
    from acoular_b200 import device as D
    rng = np.random.RandomState(11)
    x = torch.from_numpy(rng.randn(300000, 24).astype(np.float32)).pin_memory()
    ts = ac.TimeSamples(data=x, sample_freq=51200.0)
    for form in ('f64', 'tc'):
        ps = ac.PowerSpectra(source=ts, block_size=512, window='Hanning', overlap='50%', form=form)
        got = ps.csm_device.cpu().numpy()
        prec = 'complex128' if form == 'f64' else 'tc_tf32'
        ref = D.calc_csm(x.cuda(), 512, 'Hanning', '50%', prec).cpu().numpy()
        if form == 'f64':
            assert np.array_equal(got, ref)
        else:
            # FP32 accumulation per chunk of windows instead of one chunk: a few ulp(FP32) apart
            assert np.abs(got - ref).max() <= 2e-5 * np.abs(ref).max()
