"""The continuous-batching server: results alone == results in a mix; CSM running average ==
PowerSpectra over the concatenated samples; admission by HBM budget."""

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

FS = 51200.0


def _stream_specs(n=5, seed=3):
    rng = np.random.RandomState(seed)
    out = []
    for i in range(n):
        M = int(rng.choice([16, 32, 64]))
        N = int(rng.choice([256, 512, 1024]))
        side = int(rng.randint(9, 25))
        mpos = np.vstack([rng.uniform(-0.5, 0.5, (2, M)), np.zeros((1, M))])
        g = np.linspace(-0.4, 0.4, side)
        gx, gy = np.meshgrid(g, g, indexing='ij')
        gpos = np.vstack([gx.ravel(), gy.ravel(), np.full(side * side, -0.5 - 0.2 * i)])
        band = (float(rng.choice([2000.0, 4000.0, 8000.0])), 3)
        blocks = [rng.randn(5120, M).astype(np.float32) for _ in range(3)]
        out.append(dict(sid=100 + i, mpos=mpos, gpos=gpos, N=N, band=band, blocks=blocks, gshape=(side, side)))
    return out


def _open(srv, s):
    return srv.open_stream(s['sid'], s['mpos'], s['gpos'], FS, s['N'], s['band'], gshape=s['gshape'])


def test_results_alone_equal_results_in_mix():
    from acoular_b200.serving import BeamformingServer
    specs = _stream_specs()
    alone = {}
    for s in specs:
        srv = BeamformingServer()
        _open(srv, s)
        alone[s['sid']] = [srv.submit(s['sid'], b).result(timeout=60) for b in s['blocks']]
        srv.close()
    srv = BeamformingServer()
    for s in specs:
        _open(srv, s)
    futs = {s['sid']: [] for s in specs}
    for j in range(3):                      # interleave all streams' requests
        for s in specs:
            futs[s['sid']].append(srv.submit(s['sid'], s['blocks'][j]))
    mixed = {sid: [f.result(timeout=60) for f in fl] for sid, fl in futs.items()}
    assert max(srv.batches) > 1             # requests really were batched together
    srv.close()
    for s in specs:
        for a, b in zip(alone[s['sid']], mixed[s['sid']]):
            assert np.array_equal(a, b)


def test_running_csm_equals_powerspectra_over_concatenation():
    from acoular_b200.serving import BeamformingServer
    s = _stream_specs(1, seed=9)[0]
    srv = BeamformingServer()
    st = _open(srv, s)
    res = [srv.submit(s['sid'], b).result(timeout=60) for b in s['blocks']]
    srv.close()
    data = np.concatenate(s['blocks']).astype(np.float64)
    csm = O.calc_csm(data, s['N'], 'Hanning', '50%', 'complex128')
    freqs = O.fftfreq(s['N'], FS)
    bins = np.arange(st.bin_lo, st.bin_lo + st.num_bins)
    ref = O.beamformer_calc(csm, freqs, bins, O.apparent_r(s['gpos']), O.apparent_r(s['gpos'], s['mpos']), 343.0,
                            'true level', True)
    syn = O.synthetic(ref, freqs, s['band'][0], s['band'][1], s['gshape'])
    assert np.abs(res[-1] - syn).max() <= 1e-3 * np.abs(syn).max()


def test_admission_by_hbm_budget():
    from acoular_b200.serving import AdmissionError, BeamformingServer
    s = _stream_specs(1, seed=5)[0]
    srv = BeamformingServer(hbm_budget_bytes=1 << 10)
    with pytest.raises(AdmissionError):
        _open(srv, s)
    srv.close()
    srv = BeamformingServer(hbm_budget_bytes=64 << 20)
    _open(srv, s)
    used = srv.hbm_in_use
    assert used > 0
    big = np.zeros((50_000_000 // s['mpos'].shape[1], s['mpos'].shape[1]), np.float32)
    with pytest.raises(AdmissionError):
        srv.submit(s['sid'], big, block=False)
    srv.submit(s['sid'], s['blocks'][0]).result(timeout=60)
    assert srv.hbm_in_use == used           # the request's reservation was released
    srv.close_stream(s['sid'])
    assert srv.hbm_in_use == 0
    srv.close()
