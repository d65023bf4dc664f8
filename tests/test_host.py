"""CPU tests: the C-ABI library loads and exports its header, and the host-side mirror logic."""

import ctypes
import json

import numpy as np
import pytest

import acoular_b200 as ac
from acoular_b200 import _native as N
from acoular_b200 import device as D
from oracle import oracle as O


@pytest.fixture(scope='module')
def native():
    from acoular_b200 import build
    build.build()
    return N.lib()


def test_library_exports_every_header_symbol(native):
    hdr = N.header_symbols()
    assert set(hdr) == set(N.SIGNATURES), (set(hdr) ^ set(N.SIGNATURES))
    raw = ctypes.CDLL(str(N.LIB_PATH))
    for name in hdr:
        assert getattr(raw, name) is not None
    assert native.acb_abi_version() >= 1
    assert native.acb_status_string(0) == b'ok'


def test_argument_errors_are_reported_without_a_gpu(native):
    p = N.MapParams()
    p.num_mics = 1  # fewer than 2 mics
    p.num_grid = 10
    p.num_bins = 1
    p.steer_type = 3
    assert native.acb_map_f64(ctypes.byref(p), 1, 1, 1, 1, 1, None, None, None) == 1
    p.num_mics = 8
    p.steer_type = 9
    assert native.acb_map_f64(ctypes.byref(p), 1, 1, 1, 1, 1, None, None, None) == 2
    # block size beyond the FFT kernel, non power of two, window range past the samples
    assert native.acb_csm_accumulate(1, 0, 300000, 4, 131072, 65536, 0, 2, 1, 1, 0, 3, 0, 1, 1, 1 << 30, None) == 4
    assert native.acb_csm_accumulate(1, 0, 100000, 4, 1000, 500, 0, 2, 1, 1, 0, 3, 0, 1, 1, 1 << 30, None) == 1
    assert native.acb_csm_accumulate(1, 0, 1000, 4, 512, 256, 0, 4, 1, 1, 0, 3, 0, 1, 1, 1 << 30, None) == 1
    assert native.acb_csm_accumulate(1, 0, 10000, 4, 512, 256, 0, 4, 1, 1, 0, 3, 0, 1, 1, 10, None) == 5
    assert native.acb_csm_workspace_bytes(4, 3, 10, 0) == 4 * 3 * 10 * 16


def test_sincos_table_matches_host_libm(native):
    """The exception table turns correctly rounded float32 cos/sin into the C library's values."""
    tab = D.sincos_table_host()
    libm = ctypes.CDLL('libm.so.6')
    for f in (libm.cosf, libm.sinf):
        f.restype = ctypes.c_float
        f.argtypes = [ctypes.c_float]
    rng = np.random.RandomState(0)
    xs = np.concatenate([rng.uniform(0, 1500, 3000), rng.uniform(0, 4, 1000)]).astype(np.float32)
    mask = len(tab) - 1
    n_exc = 0
    for x in xs:
        key = int(x.view(np.uint32))
        slot = ((key * 0x9E3779B97F4A7C15) & (2 ** 64 - 1)) >> 20
        dc = ds = 0
        for p in range(64):
            e = int(tab[(slot + p) & mask])
            if e == 2 ** 64 - 1:
                break
            if e >> 32 == key:
                dc, ds = int(np.int8(np.uint8((e >> 8) & 0xFF))), int(np.int8(np.uint8(e & 0xFF)))
                n_exc += 1
                break
        c = np.float32(np.cos(np.float64(x)))
        s = np.float32(np.sin(np.float64(x)))
        c = (c.view(np.int32) + np.int32(dc)).view(np.float32)
        s = (s.view(np.int32) + np.int32(ds)).view(np.float32)
        assert c == np.float32(libm.cosf(float(x))) and s == np.float32(libm.sinf(float(x)))


def test_rect_grid_matches_reference_layout():
    g = ac.RectGrid(x_min=-0.2, x_max=0.2, y_min=-0.2, y_max=0.2, z=-0.3, increment=0.01)
    pos, shape = O.rect_grid_pos(-0.2, 0.2, -0.2, 0.2, -0.3, 0.01)
    assert g.shape == shape == (41, 41)
    assert np.array_equal(g.pos, pos)
    g3 = ac.RectGrid3D(x_min=-0.2, x_max=0.2, y_min=-0.2, y_max=0.2, z_min=0.5, z_max=0.9, increment=0.2)
    pos3, shape3 = O.rect_grid3d_pos(-0.2, 0.2, -0.2, 0.2, 0.5, 0.9, 0.2)
    assert g3.shape == shape3 and np.array_equal(g3.pos, pos3)
    assert g.indices(-0.1, -0.1, 0.1, 0.1) == (np.s_[10:31], np.s_[10:31])
    xi, yi = g.indices(0.0, 0.0, 0.025)
    assert len(xi) == len(yi) == 21  # points within 2.5 increments of the centre


@pytest.mark.parametrize('S,N,ov', [(2000, 128, 2), (51200, 128, 2), (100, 128, 1), (1000, 256, 8), (4096, 1024, 4)])
def test_window_count_matches_generator(S, N, ov):
    assert D.num_windows(S, N, ov) == sum(1 for _ in O.source_windows(np.zeros((S, 1)), N, ov))
    assert D.num_blocks(S, N, ov) == O.num_blocks(S, N, ov)


def test_power_spectra_settings_validation():
    ts = ac.TimeSamples(data=np.zeros((1000, 4)), sample_freq=51200)
    ps = ac.PowerSpectra(source=ts, block_size=128, window='Blackman')
    assert np.array_equal(ps.fftfreq(), O.fftfreq(128, 51200.0))
    assert ps.fftfreq()[20] == 8000.0
    with pytest.raises(ValueError):
        ps.block_size = 100
    with pytest.raises(ValueError):
        ps.window = 'Kaiser'
    with pytest.raises(ValueError):
        ps.overlap = '33%'
    ps.overlap = '50%'
    assert ps.num_blocks == O.num_blocks(1000, 128, 2)
    ps.ind_low, ps.ind_high = 3, 10
    assert list(ps.indices) == list(range(3, 10))


def test_beamformer_settings_and_channel_check():
    mg = ac.MicGeom(pos_total=np.random.RandomState(0).randn(3, 5))
    ts = ac.TimeSamples(data=np.zeros((1000, 4)), sample_freq=51200)
    ps = ac.PowerSpectra(source=ts, block_size=128)
    st = ac.SteeringVector(grid=ac.RectGrid(increment=0.5), mics=mg)
    bb = ac.BeamformerBase(freq_data=ps, steer=st)
    with pytest.raises(ValueError, match='4 channels do not fit 5 mics'):
        bb.result  # noqa: B018
    assert bb.sig_loss_norm() == 4 / 3  # num_channels / (num_channels - 1)
    bb.r_diag_norm = 2.0
    assert bb.sig_loss_norm() == 2.0
    bb.r_diag = False
    assert bb.sig_loss_norm() == 1.0
    with pytest.raises(ValueError):
        ac.SteeringVector(steer_type='foo')
    with pytest.raises(ValueError):
        ac.BeamformerBase(form='gpu')
    for prec in ('bf16x3', 'tf32', 'fp16'):
        assert ac.BeamformerBase(form='tc', tc_precision=prec).tc_precision == prec
    with pytest.raises(ValueError, match='tc_precision'):
        ac.BeamformerBase(form='tc', tc_precision='fp8')


def test_band_indices_match_reference_rule():
    freqs = O.fftfreq(128, 51200.0)
    assert O.band_indices(freqs, 8000.0, 3) == (18, 23)


def test_steering_host_helpers_match_oracle():
    mg = ac.MicGeom(pos_total=np.random.RandomState(1).normal(size=15).reshape(3, 5))
    g = ac.ImportGrid(pos=np.array([[0.0], [0.0], [1.0]]))
    st = ac.SteeringVector(grid=g, mics=mg)
    np.testing.assert_allclose(st.rm, O.apparent_r(g.pos, mg.pos), rtol=1e-15)
    np.testing.assert_allclose(st.r0, O.apparent_r(g.pos), rtol=1e-15)
    st.ref = 2.5
    assert np.array_equal(st.r0, np.full(1, 2.5))
    tr = st.transfer(2000.0)
    assert tr.shape == (1, 5)


def test_l_p_and_integrate():
    x = np.array([[4e-10, 0.0], [-1.0, 4e-8]])
    np.testing.assert_allclose(ac.L_p(x), O.L_p(x))
    g = ac.RectGrid(x_min=-1, x_max=1, y_min=-1, y_max=1, z=1, increment=1.0)
    data = np.arange(9.0)
    assert ac.integrate(data, g, (-1, -1, 0, 0)) == data.reshape(3, 3)[0:2, 0:2].sum()
    h = ac.integrate(np.vstack([data, 2 * data]), g, (0, 0, 1, 1))
    assert np.array_equal(h, [data.reshape(3, 3)[1:, 1:].sum(), 2 * data.reshape(3, 3)[1:, 1:].sum()])


def test_autotune_classes_and_lookup(tmp_path):
    from acoular_b200 import autotune as A
    assert A.mic_bucket(2) == 32 and A.mic_bucket(33) == 64 and A.mic_bucket(1024) == 1024
    assert A.mic_bucket(5000) == 2048
    assert A.item_bucket(128 * 37, 1) == 'tiny' and A.item_bucket(128 * 38, 1) == 'few'
    assert A.item_bucket(128 * 148, 1) == 'few' and A.item_bucket(128 * 149, 1) == 'mid'
    assert A.item_bucket(160801, 513) == 'many'
    # candidates: distinct schedules only, splits never above the pass count
    for M in (2, 40, 256, 600, 2048):
        C = (M + 15) // 16
        cands = A.candidates(M)
        assert (16, 1) in cands or (C <= 4 and cands[0][1] == 1)
        for pw, sp in cands:
            assert pw in A.PASS_CHUNKS and 1 <= sp <= -(-C // pw)
    assert A.candidates(32) == [(4, 1)]
    # missing table -> default; a table entry is honoured; an invalid one falls back
    missing = tmp_path / 'none.json'
    assert A.lookup(256, 160801, 513, 'bf16x3', path=missing) == A.DEFAULT
    t = tmp_path / 't.json'
    key = A.shape_class(600, 1000, 2, 'tf32')
    t.write_text(json.dumps({'classes': {key: {'pass_chunks': 8, 'splits': 4}}}))
    assert A.lookup(600, 1000, 2, 'tf32', path=t) == (8, 4)
    t2 = tmp_path / 't2.json'
    t2.write_text(json.dumps({'classes': {key: {'pass_chunks': 8, 'splits': 8}}}))   # 5 passes < 8
    assert A.lookup(600, 1000, 2, 'tf32', path=t2) == A.DEFAULT


def test_committed_tuning_table_is_valid():
    from acoular_b200 import autotune as A
    if not A.TABLE_PATH.exists():
        pytest.skip('no tuning table')
    tab = json.loads(A.TABLE_PATH.read_text())
    assert tab['classes']
    for key, ent in tab['classes'].items():
        prec, mb, ib = key.split(':')
        M = int(mb[1:])
        assert prec in ('bf16x3', 'tf32', 'fp16') and ib in ('tiny', 'few', 'mid', 'many')
        assert (ent['pass_chunks'], ent['splits']) in A.candidates(M)
        assert ent['ms'] == min(ent['candidates_ms'].values())


def test_noalloc_entry_point_argument_codes_match_workspace_entry_point():
    """acb_map_tc_noalloc reports argument errors with acb_map_tc's status codes (the checks return before
    any CUDA call, so this runs without a GPU); a valid request beyond its fixed array is ACB_ERR_SHAPE."""
    import ctypes

    from acoular_b200 import _native as N
    from acoular_b200 import build
    from acoular_b200 import device as D
    build.build()
    L = N.lib()

    def both(p, prec, csm=1):
        a = L.acb_map_tc(ctypes.byref(p), prec, csm, 1, 1, 1, 1, None, None, 0, None, None)
        b = L.acb_map_tc_noalloc(ctypes.byref(p), prec, csm, 1, 1, 1, 1, None, None, None)
        return a, b

    ok = D.map_params(64, 1000, 4, 'true level', True, 1.0)
    assert both(ok, 7) == (N.ACB_ERR_UNSUPPORTED, N.ACB_ERR_UNSUPPORTED)     # unknown precision
    assert both(ok, 0, csm=None) == (N.ACB_ERR_ARG, N.ACB_ERR_ARG)           # null CSM
    for bad, code in (({'steer_type': 9}, N.ACB_ERR_ARG), ({'num_mics': 4096}, N.ACB_ERR_UNSUPPORTED),
                      ({'num_bins': 0}, N.ACB_ERR_SHAPE), ({'num_grid': 0}, N.ACB_ERR_SHAPE),
                      ({'tc_pass_chunks': 5}, N.ACB_ERR_ARG)):
        p = D.map_params(64, 1000, 4, 'true level', True, 1.0)
        for k, v in bad.items():
            setattr(p, k, v)
        assert both(p, 0) == (code, code), bad
    big = D.map_params(256, 1000, 100, 'classic', True, 1.0)                 # 100 bins x 544 KB > 32 MiB
    assert L.acb_map_tc_noalloc(ctypes.byref(big), 0, 1, 1, 1, 1, 1, None, None, None) == N.ACB_ERR_SHAPE


def test_heevd_select_size_rule():
    """The selected-eigenpair solver's size rule (its work arrays in 200 KB of shared memory): BeamformerEig
    takes the full decomposition beyond it."""
    from acoular_b200 import device as D
    assert D.heevd_select_supported(1, 1) and D.heevd_select_supported(256, 1) and D.heevd_select_supported(3000, 1)
    assert not D.heevd_select_supported(3200, 1) and not D.heevd_select_supported(4097, 1)
    assert D.heevd_select_supported(256, 4) and not D.heevd_select_supported(256, 5)
    assert not D.heevd_select_supported(2, 3)


def test_map_launch_sizes():
    """BeamformerBase's launch plan: every bin once, in order, no launch above the memory cap, and for the
    513-bin workload a last launch of a few bins (the download left after the computation)."""
    from acoular_b200.fbeamform import _launch_sizes
    for n in (1, 2, 3, 5, 8, 64, 65, 513, 1000):
        for cap in (1, 7, 30, 10**9):
            sizes = _launch_sizes(n, cap)
            assert sum(sizes) == n and min(sizes) >= 1 and max(sizes) <= cap
    s = _launch_sizes(513, 10**9)
    assert s[-1] <= 4 and len(s) <= 12
    # the 256-mic workload's maps (401 x 401 points, 8 bytes) keep the overlapped plan; a band of 5 bins on a
    # 41 x 41 grid is one launch, and a cap still splits it
    assert _launch_sizes(513, 10**9, 160801 * 8) == s
    assert _launch_sizes(5, 10**9, 1681 * 8) == [5]
    assert _launch_sizes(5, 2, 1681 * 8) == [2, 2, 1]


def test_time_samples_digest():
    """TimeSamples' content digest: equal for equal samples (another array object), different when a sampled
    row, the last row, the shape or the sample rate differs; numpy and torch data both work."""
    import torch

    import acoular_b200 as ac
    a = np.random.RandomState(3).randn(51200, 64)
    d = ac.TimeSamples(data=a, sample_freq=51200.0).digest
    assert ac.TimeSamples(data=a.copy(), sample_freq=51200.0).digest == d
    b = a.copy()
    b[0, 5] += 1.0
    assert ac.TimeSamples(data=b, sample_freq=51200.0).digest != d
    b = a.copy()
    b[-1, 0] += 1.0
    assert ac.TimeSamples(data=b, sample_freq=51200.0).digest != d
    assert ac.TimeSamples(data=a[:-1], sample_freq=51200.0).digest != d
    assert ac.TimeSamples(data=a, sample_freq=48000.0).digest != d
    t = torch.from_numpy(a)
    assert ac.TimeSamples(data=t, sample_freq=51200.0).digest == ac.TimeSamples(data=t.clone(), sample_freq=51200.0).digest
    for empty in (np.zeros((0, 4)), np.arange(10.0)):
        assert ac.TimeSamples(data=empty, sample_freq=1.0).digest.startswith('_')
