"""Tensor-core (split-BF16, tcgen05) map against the FP64 oracle.

Error measure (the one the benchmark reports): max |map - ref| / max |ref| over the map, per call,
and the peak level error in dB.  Bar: <= 1e-3 relative and <= 0.05 dB at the peak.
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

STEERS = ['classic', 'inverse', 'true level', 'true location']
TOL = 1e-3


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _case(M, G, seed, nb=3, z=-0.6):
    rng = np.random.RandomState(seed)
    mpos = np.vstack([rng.uniform(-0.5, 0.5, (2, M)), np.zeros((1, M))])
    gpos = np.vstack([rng.uniform(-0.4, 0.4, (2, G)), np.full((1, G), z)])
    # CSM of a few coherent sources plus noise (peaked maps, like the benchmark data)
    src = np.vstack([rng.uniform(-0.3, 0.3, (2, 3)), np.full((1, 3), z)])
    freqs = np.array([1500.0, 4000.0, 9100.0, 12000.0])[:nb]
    csm = np.zeros((nb, M, M), complex)
    for f_i, f in enumerate(freqs):
        k = 2 * np.pi * f / 343.0
        for s in range(3):
            r = O.apparent_r(src[:, s:s + 1], mpos).reshape(-1)
            a = np.exp(-1j * k * r) / r
            csm[f_i] += (1.0 + s) * np.outer(a, a.conj())
        X = rng.randn(2 * M, M) + 1j * rng.randn(2 * M, M)
        csm[f_i] += 0.05 * np.abs(csm[f_i]).max() * (X.conj().T @ X) / (2 * M)
    return mpos, gpos, freqs, csm


def _tc(csm, freqs, mpos, gpos, steer, r_diag, ref=None, precision='bf16x3'):
    from acoular_b200 import device as D
    dev = torch.device('cuda')
    M = mpos.shape[1]
    out = D.map_tc(torch.as_tensor(csm, device=dev), torch.as_tensor(2 * np.pi * freqs / 343.0, device=dev),
                   torch.as_tensor(mpos, device=dev), torch.as_tensor(np.ascontiguousarray(gpos), device=dev), steer,
                   r_diag, O.sig_loss_norm(r_diag, M), ref=ref, clip_negative=r_diag, precision=precision)
    return out.cpu().numpy()


@pytest.mark.parametrize('M,G', [(2, 1), (16, 128), (37, 300), (64, 257), (128, 129), (256, 200), (300, 150),
                                 (513, 140)])
@pytest.mark.parametrize('steer', STEERS)
def test_tc_vs_oracle(M, G, steer):
    mpos, gpos, freqs, csm = _case(M, G, seed=M + G)
    r0, rm = O.apparent_r(gpos), O.apparent_r(gpos, mpos)
    for r_diag in (False, True):
        ref = O.beamformer_calc(csm, freqs, range(len(freqs)), r0, rm, 343.0, steer, r_diag)
        got = _tc(csm, freqs, mpos, gpos, steer, r_diag)
        for b in range(len(freqs)):
            assert rel(got[b], ref[b]) <= TOL, (b, rel(got[b], ref[b]))


def test_tc_config1_golden_and_peak_level(golden):
    from acoular_b200 import workloads
    d = golden('config1_band.npz')
    wl = workloads.three_sources_64()
    for steer in STEERS:
        for r_diag in (False, True):
            key = f'map_{steer.replace(" ", "_")}_{int(r_diag)}'
            got = _tc(d['csm_band'], d['freqs'][18:23], wl.mics.pos, wl.grid.pos, steer, r_diag)
            assert rel(got, d[key]) <= TOL
            syn, ref = got.sum(0), d['syn_' + key].reshape(-1)
            assert rel(syn, ref) <= TOL
            assert abs(O.L_p(syn.max()) - O.L_p(ref.max())) <= 0.05


def test_tc_reference_position_and_workspace_errors():
    from acoular_b200 import _native as N
    from acoular_b200 import device as D
    mpos, gpos, freqs, csm = _case(24, 150, seed=3)
    ref_pt = np.array([0.05, 0.1, -0.02])
    r0, rm = O.apparent_r(gpos, ref_pt[:, None]), O.apparent_r(gpos, mpos)
    ref = O.beamformer_calc(csm, freqs, range(3), r0, rm, 343.0, 'true level', True)
    got = _tc(csm, freqs, mpos, gpos, 'true level', True, ref=ref_pt)
    assert rel(got, ref) <= TOL
    p = D.map_params(3000, 10, 1, 'classic', True, 1.0)
    import ctypes
    assert N.lib().acb_map_tc(ctypes.byref(p), 0, 1, 1, 1, 1, 1, None, 1, 1 << 40, None, None) == 4  # > 2048 mics
    p = D.map_params(64, 10, 1, 'classic', True, 1.0)
    assert N.lib().acb_map_tc(ctypes.byref(p), 0, 1, 1, 1, 1, 1, None, 1, 10, None, None) == 5  # workspace


def test_tc_error_word_stays_clear():
    from acoular_b200 import device as D
    dev = torch.device('cuda')
    mpos, gpos, freqs, csm = _case(64, 1000, seed=9)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    D.map_tc(torch.as_tensor(csm, device=dev), torch.as_tensor(2 * np.pi * freqs / 343.0, device=dev),
             torch.as_tensor(mpos, device=dev), torch.as_tensor(gpos, device=dev), 'classic', True, 1.0,
             error_word=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0


@pytest.mark.parametrize('precision', ['bf16x3', 'fp16'])
@pytest.mark.parametrize('M,G,nb', [(64, 20000, 4), (256, 12000, 3), (40, 50000, 2), (700, 2000, 2)])
def test_tc_persistent_many_items_per_cta(M, G, nb, precision):
    """More work items (bin x 128-point tile) than CTAs: the pipeline runs across item boundaries (FP16:
    chunk-pair steps, an odd chunk count per pass at 40 and 700 mics)."""
    mpos, gpos, freqs, csm = _case(M, G, seed=M * 3 + nb, nb=nb)
    r0, rm = O.apparent_r(gpos), O.apparent_r(gpos, mpos)
    ref = O.beamformer_calc(csm, freqs, range(nb), r0, rm, 343.0, 'true location', True)
    got = _tc(csm, freqs, mpos, gpos, 'true location', True, precision=precision)
    for b in range(nb):
        assert rel(got[b], ref[b]) <= TOL


@pytest.mark.parametrize('precision', ['tf32', 'bf16x3', 'fp16'])
@pytest.mark.parametrize('M', [16, 32])
def test_tc_short_items_many_per_cta(M, precision):
    """Items of one or two steps (<= 32 mics), many per CTA: the steering warps run more than an item
    ahead of the epilogue, and the per-item normalisation sums must still reach the right item."""
    from acoular_b200 import device as D
    dev = torch.device('cuda')
    nb = 4
    mpos, gpos, freqs, csm = _case(M, 40000, seed=M + 1, nb=nb)
    r0, rm = O.apparent_r(gpos), O.apparent_r(gpos, mpos)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    for steer in ('true level', 'inverse'):
        ref = O.beamformer_calc(csm, freqs, range(nb), r0, rm, 343.0, steer, True)
        for tuning in ('auto', None):
            out = D.map_tc(torch.as_tensor(csm, device=dev), torch.as_tensor(2 * np.pi * freqs / 343.0, device=dev),
                           torch.as_tensor(mpos, device=dev), torch.as_tensor(gpos, device=dev), steer, True,
                           O.sig_loss_norm(True, M), clip_negative=True, precision=precision, error_word=err,
                           tuning=tuning)
            torch.cuda.synchronize()
            assert int(err.item()) == 0
            got = out.cpu().numpy()
            for b in range(nb):
                assert rel(got[b], ref[b]) <= TOL, (steer, tuning, b, rel(got[b], ref[b]))


def _instances(specs, seed=0):
    """Uneven instances (M, G, bins) with random geometry and CSMs, as device tensors."""
    from acoular_b200 import device as D
    dev = torch.device('cuda')
    out = []
    for idx, (M, G, nb) in enumerate(specs):
        mpos, gpos, freqs, csm = _case(M, G, seed=seed + 17 * idx, nb=nb, z=-0.5 - 0.1 * idx)
        out.append((D.MapInstance(torch.as_tensor(csm, device=dev),
                                  torch.as_tensor(2 * np.pi * freqs / 343.0, device=dev),
                                  torch.as_tensor(mpos, device=dev), torch.as_tensor(gpos, device=dev),
                                  'true level', True, O.sig_loss_norm(True, M)), (mpos, gpos, freqs, csm)))
    return out


@pytest.mark.parametrize('precision', ['bf16x3', 'fp16'])
def test_tc_batch_uneven_instances_equal_alone(precision):
    """Each instance's map is the same in the batched launch as alone, and matches the oracle."""
    from acoular_b200 import device as D
    specs = [(32, 441, 3), (64, 2000, 2), (128, 700, 4), (256, 300, 2), (300, 150, 2), (37, 90001, 1),
             (32, 40000, 4), (16, 20000, 3)]
    inst = _instances(specs)
    err = torch.zeros(1, dtype=torch.int32, device=inst[0][0].csm.device)
    D.map_tc_batch([i for i, _ in inst], precision=precision, error_word=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    for it, (mpos, gpos, freqs, csm) in inst:
        alone = D.map_tc(it.csm, it.wavenumbers, it.mpos, it.gpos, 'true level', True, it.norm,
                         precision=precision).cpu().numpy()
        got = it.out.cpu().numpy()
        assert np.array_equal(got, alone)
        nb = len(freqs)
        if gpos.shape[1] <= 2000:
            ref = O.beamformer_calc(csm, freqs, range(nb), O.apparent_r(gpos), O.apparent_r(gpos, mpos), 343.0,
                                    'true level', True)
            assert rel(got, ref) <= TOL


def test_tc_batch_graph_capture_replay():
    from acoular_b200 import device as D
    inst = _instances([(64, 3000, 3), (128, 1000, 2)], seed=5)
    its = [i for i, _ in inst]
    D.map_tc_batch(its)  # warm-up outside capture (workspace allocation, kernel attributes)
    torch.cuda.synchronize()
    ref = [it.out.clone() for it in its]
    for it in its:
        it.out.zero_()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        D.map_tc_batch(its)
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    for it, r in zip(its, ref):
        assert torch.equal(it.out, r)


@pytest.mark.parametrize('precision', ['tf32', 'fp16'])
@pytest.mark.parametrize('M,G', [(16, 128), (64, 257), (256, 200), (300, 150)])
@pytest.mark.parametrize('steer', STEERS)
def test_tf32_form_vs_oracle(M, G, steer, precision):
    """The single-product operand forms (FP32 rounded to TF32; FP16 with R' scaled per bin), FP32
    accumulation; <= 1e-3 of max."""
    mpos, gpos, freqs, csm = _case(M, G, seed=M + 3 * G)
    r0, rm = O.apparent_r(gpos), O.apparent_r(gpos, mpos)
    for r_diag in (False, True):
        ref = O.beamformer_calc(csm, freqs, range(len(freqs)), r0, rm, 343.0, steer, r_diag)
        got = _tc(csm, freqs, mpos, gpos, steer, r_diag, precision=precision)
        for b in range(len(freqs)):
            assert rel(got[b], ref[b]) <= TOL, (b, rel(got[b], ref[b]))


@pytest.mark.parametrize('scale', [1e-30, 1e-8, 1.0, 1e12, 1e40])
def test_fp16_form_per_bin_scale(scale):
    """FP16 operands keep their precision whatever the CSM's magnitude: each bin's R' is scaled by a
    power of two, here with bins 1e6 apart inside one call and the whole CSM from 1e-30 to 1e40."""
    mpos, gpos, freqs, csm = _case(64, 500, seed=7)
    csm = csm * (scale * np.array([1.0, 1e6, 1e-6])[:, None, None])
    r0, rm = O.apparent_r(gpos), O.apparent_r(gpos, mpos)
    for steer in ('true level', 'classic'):
        ref = O.beamformer_calc(csm, freqs, range(len(freqs)), r0, rm, 343.0, steer, True)
        got = _tc(csm, freqs, mpos, gpos, steer, True, precision='fp16')
        for b in range(len(freqs)):
            assert rel(got[b], ref[b]) <= TOL, (b, rel(got[b], ref[b]))


def test_fp16_form_range_error_bit():
    """'inverse' steering weights are the distances themselves: grid points 1e5 m away give FP16
    operands above 65504, which the launch reports in bit 1 of the error word (the map holds
    non-finite values there) instead of returning a wrong finite map."""
    from acoular_b200 import device as D
    dev = torch.device('cuda')
    mpos, gpos, freqs, csm = _case(32, 300, seed=8)
    far = gpos.copy()
    far[2] = -1e5
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    args = (torch.as_tensor(csm, device=dev), torch.as_tensor(2 * np.pi * freqs / 343.0, device=dev),
            torch.as_tensor(mpos, device=dev))
    D.map_tc(*args, torch.as_tensor(gpos, device=dev), 'inverse', True, 1.0, precision='fp16', error_word=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    out = D.map_tc(*args, torch.as_tensor(far, device=dev), 'inverse', True, 1.0, precision='fp16',
                   error_word=err)
    torch.cuda.synchronize()
    assert int(err.item()) & 2
    assert not np.isfinite(out.cpu().numpy()).all()


@pytest.mark.parametrize('precision', ['bf16x3', 'fp16'])
@pytest.mark.parametrize('M,G,steer', [(40, 700, 'true level'), (256, 300, 'true location'), (600, 260, 'inverse'),
                                       (1100, 130, 'classic')])
def test_tc_tile_width_and_split_agree(M, G, steer, precision):
    """Every (pass width, split) candidate gives the default schedule's map (FP64 partial-sum order
    differs only), and the single-instance entry (acb_map_tc) gives it too."""
    from acoular_b200 import autotune
    from acoular_b200 import device as D
    dev = torch.device('cuda')
    mpos, gpos, freqs, csm = _case(M, G, seed=M + 5 * G)
    args = (torch.as_tensor(csm, device=dev), torch.as_tensor(2 * np.pi * freqs / 343.0, device=dev),
            torch.as_tensor(mpos, device=dev), torch.as_tensor(np.ascontiguousarray(gpos), device=dev), steer, True,
            O.sig_loss_norm(True, M))
    base = D.map_tc(*args, clip_negative=True, tuning=(16, 1), precision=precision).cpu().numpy()
    single = D.map_tc(*args, clip_negative=True, tuning=None, precision=precision).cpu().numpy()
    assert np.array_equal(single, base)
    cands = autotune.candidates(M)
    assert len(cands) >= (3 if M > 64 else 1)
    for pw, sp in cands:
        got = D.map_tc(*args, clip_negative=True, tuning=(pw, sp), precision=precision).cpu().numpy()
        assert rel(got, base) <= 1e-12, (pw, sp)
    ref = O.beamformer_calc(csm, freqs, range(len(freqs)), O.apparent_r(gpos), O.apparent_r(gpos, mpos), 343.0, steer,
                            True)
    assert rel(base, ref) <= TOL


def test_tc_split_graph_replay_and_mix():
    """Split instances replay in a CUDA graph (group counters are reset by every launch) and give the
    same map inside a batch with unsplit instances."""
    from acoular_b200 import device as D
    inst = _instances([(600, 700, 2), (64, 3000, 3), (300, 500, 2)], seed=11)
    its = [i for i, _ in inst]
    its[0].tuning, its[1].tuning, its[2].tuning = (4, 8), (16, 1), (8, 2)
    alone = []
    for it in its:
        D.map_tc_batch([it])
        alone.append(it.out.clone())
    D.map_tc_batch(its)
    torch.cuda.synchronize()
    for it, a in zip(its, alone):
        assert torch.equal(it.out, a)
        it.out.zero_()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        D.map_tc_batch(its)
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    for it, a in zip(its, alone):
        assert torch.equal(it.out, a)


@pytest.fixture(scope='module')
def precision256_reduced():
    """The 256-mic workload's geometry and sources (256 mics in a 1 m disk, 8 monopoles at z = -1 m, 10 s
    at 51.2 kHz, block 1024, Hanning, 50 %) with its grid reduced to 101 x 101 points over [-1, 1]^2 and
    8 bins spread over the band; the complex128 CSM comes from the device path (itself pinned to the
    oracle to 1e-12 elsewhere) and is handed to the oracle as is."""
    from acoular_b200 import device as D
    from acoular_b200 import workloads
    from acoular_b200.grids import RectGrid
    wl = workloads.precision_256()
    dev = torch.device('cuda')
    x = workloads.monopole_time_data_torch(wl, device=dev)
    N = wl.block_size
    bins = np.array([20, 80, 150, 220, 290, 360, 430, 500])
    csm = D.calc_csm(x, N, 'Hanning', '50%', 'complex128')[torch.as_tensor(bins, device=dev)].contiguous()
    del x
    grid = RectGrid(x_min=-1.0, x_max=1.0, y_min=-1.0, y_max=1.0, z=-1.0, increment=0.02)
    freqs = np.abs(np.fft.fftfreq(N, 1 / wl.fs)[bins])
    return wl.mics.pos, grid.pos, freqs, csm.cpu().numpy()


@pytest.mark.parametrize('precision', ['tf32', 'bf16x3', 'fp16'])
@pytest.mark.parametrize('steer', STEERS)
def test_precision_matrix_256mic_reduced_grid(precision256_reduced, steer, precision):
    """The precision matrix of the 256-mic workload at a reduced size: each steering type x r_diag x
    tensor-core precision against the FP64 oracle, <= 1e-3 of max and <= 0.05 dB at each bin's peak."""
    mpos, gpos, freqs, csm = precision256_reduced
    assert gpos.shape[1] == 101 * 101
    r0, rm = O.apparent_r(gpos), O.apparent_r(gpos, mpos)
    nb = len(freqs)
    for r_diag in (True, False):
        ref = O.beamformer_calc(csm, freqs, range(nb), r0, rm, 343.0, steer, r_diag)
        got = _tc(csm, freqs, mpos, gpos, steer, r_diag, precision=precision)
        for b in range(nb):
            assert rel(got[b], ref[b]) <= TOL, (b, r_diag, rel(got[b], ref[b]))
            pk = ref[b].argmax()
            assert abs(O.L_p(got[b][pk:pk + 1]) - O.L_p(ref[b][pk:pk + 1]))[0] <= 0.05
