"""RFFT / AutoPowerSpectra / CrossPowerSpectra on the GPU (acb_spectra, acb_auto_spectra,
acb_cross_spectra) against the reference's generators (tests/golden/fprocess_kat.npz).

Tolerances: the spectra come from an FP64 FFT of another radix order than scipy's, so complex128 values
agree to <= 1e-12 of each block's max; complex64 / float32 values are the same numbers rounded, within
one float32 ulp of the max (2e-7 of max).  Block structure (sizes, the zero row of an empty source)
is exact.
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _close(got, ref, tol):
    ref = np.asarray(ref)
    assert got.shape == ref.shape and got.dtype == ref.dtype, (got.shape, ref.shape, got.dtype, ref.dtype)
    assert np.abs(got.astype(np.complex128) - ref).max() <= tol * np.abs(ref).max()


def _tol(dtype):
    return 2e-7 if np.dtype(dtype) in (np.complex64, np.float32) else 1e-12


@pytest.fixture(scope='module')
def src(golden):
    import acoular_b200 as ac
    s = golden('small_kat.npz')
    return ac.TimeSamples(data=s['data'], sample_freq=float(s['fs'])), s


@pytest.mark.parametrize('ci', range(4))
def test_rfft_auto_cross_vs_reference(golden, src, ci):
    import acoular_b200 as ac
    g = golden('fprocess_kat.npz')
    ts, s = src
    bs, win, ov, prec, scaling, num = g[f'rfft{ci}_case']
    bs, num = int(bs), int(num)
    rf = ac.RFFT(source=ts, block_size=bs, window=win, overlap=ov, precision=prec, scaling=scaling)
    assert rf.num_freqs == bs // 2 + 1 and rf.num_samples == s['data'].shape[0] // bs
    blocks = list(rf.result(num))
    assert [b.shape[0] for b in blocks] == list(g[f'rfft{ci}_sizes'])
    _close(np.concatenate(blocks), g[f'rfft{ci}'], _tol(prec))
    for ai, (sc, ss, ap) in enumerate([('power', True, 'float64'), ('psd', False, 'float32')]):
        aps = ac.AutoPowerSpectra(source=rf, scaling=sc, single_sided=ss, precision=ap)
        got = np.concatenate(list(aps.result(num)))
        ref = g[f'aps{ci}_{ai}']
        assert got.dtype == ref.dtype
        # float64 output of complex64 spectra holds float32 products, like the reference's
        tol = 2e-7 if (prec == 'complex64' or ap == 'float32') else 1e-12
        assert np.abs(got - ref).max() <= tol * np.abs(ref).max()
    cprec = 'complex64' if prec == 'complex64' else 'complex128'
    cps = ac.CrossPowerSpectra(source=rf, scaling='psd' if ci % 2 else 'power', precision=cprec)
    assert cps.num_channels == 64
    cb = list(cps.result(num))
    assert [b.shape[0] for b in cb] == list(g[f'cps{ci}_sizes'])
    allc = np.concatenate(cb)
    _close(allc[:2 * num], g[f'cps{ci}'], _tol(cprec))
    ref_sum = g[f'cps{ci}_sum']
    assert np.abs(allc.astype(np.complex128).sum(axis=0) - ref_sum).max() <= 10 * _tol(cprec) * np.abs(ref_sum).max()


def test_device_chain_and_welch_property(src):
    """RFFT -> CrossPowerSpectra stays on the device; summed over all snapshots (scaled back) it is the
    Welch CSM of PowerSpectra on the same windows."""
    import acoular_b200 as ac
    ts, s = src
    rf = ac.RFFT(source=ts, block_size=128, window='Hanning', overlap='50%')
    cps = ac.CrossPowerSpectra(source=rf)
    dev_blocks = list(cps.result_device(8))
    assert all(b.is_cuda and b.shape[1:] == (65, 8, 8) for b in dev_blocks)
    host_blocks = list(cps.result(8))
    for d, h in zip(dev_blocks, host_blocks):
        np.testing.assert_array_equal(d.cpu().numpy().reshape(d.shape[0], -1), h)
    total = torch.cat(dev_blocks).sum(dim=0).cpu().numpy()
    ps = ac.PowerSpectra(source=ts, block_size=128, window='Hanning', overlap='50%')
    w = np.hanning(128)
    svalue = 1 / np.sqrt(np.dot(w, w) / 128)
    # RFFT scales spectra by svalue (power scale 2/N^2); PowerSpectra divides the Welch sum by
    # N * sum(w^2) * num_blocks / 2
    welch = total / (svalue**2 * 2 / 128**2) * 2 / (128 * np.dot(w, w) * ps.num_blocks)
    csm = ps.csm
    assert np.abs(welch - csm).max() <= 1e-12 * np.abs(csm).max()


def test_edge_cases(src):
    import acoular_b200 as ac
    ts, s = src
    short = ac.TimeSamples(data=s['data'][:100], sample_freq=float(s['fs']))
    rf = ac.RFFT(source=short, block_size=128)
    blocks = list(rf.result(4))          # no complete block: one zero row, as the reference yields
    assert len(blocks) == 1 and blocks[0].shape == (1, 65 * 8) and not blocks[0].any()
    assert list(rf.result(1)) == []
    with pytest.raises(ValueError):
        ac.RFFT(source=ts, block_size=127)
    with pytest.raises(ValueError):
        next(ac.RFFT(source=ts, block_size=96).result(2))
    with pytest.raises(ValueError):
        next(ac.CrossPowerSpectra(source=ac.RFFT(source=ts, block_size=64), calc_mode='upper').result(2))
    one = ac.TimeSamples(data=s['data'][:, :1].copy(), sample_freq=float(s['fs']))
    rf1 = ac.RFFT(source=one, block_size=64)
    up = np.concatenate(list(ac.CrossPowerSpectra(source=rf1, calc_mode='upper').result(5)))
    full = np.concatenate(list(ac.CrossPowerSpectra(source=rf1).result(5)))
    np.testing.assert_array_equal(up, full)
    spec = np.concatenate(list(rf1.result(5)))
    ref = np.concatenate(list(O.cross_power_blocks([spec], 33, 1, O.power_scale(64, float(s['fs']), 'power', True),
                                                   'complex128')))
    assert np.abs(full - ref).max() <= 1e-13 * np.abs(ref).max()


def test_rfft_large_block():
    """RFFT with a 32768-sample block (sub-transforms of 8192 points and a combining pass) against the
    oracle's generator, complex128 at 1e-12 of each block's max."""
    import acoular_b200 as ac
    rng = np.random.RandomState(11)
    data = rng.randn(3 * 32768, 3)
    ts = ac.TimeSamples(data=data, sample_freq=48000.0)
    rf = ac.RFFT(source=ts, block_size=32768, window='Hanning', overlap='50%', scaling='amplitude')
    got = list(rf.result(2))
    ref = list(O.rfft_blocks(data, 32768, 'Hanning', '50%', 'complex128', 'amplitude', 2))
    assert [b.shape for b in got] == [b.shape for b in ref]
    for a, b in zip(got, ref):
        _close(a, b, 1e-12)
