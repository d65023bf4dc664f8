"""Tensor-core CSM (TF32 / split-BF16 Gram on tcgen05) against the FP64 CSM of the same samples.

The FP64 path is pinned to the reference (tests/test_gpu_plain.py); here the tensor-core Welch sums
must agree with it to the operand precision: TF32 rounds each spectrum value to 2^-11 relative,
split BF16 (hi + lo, three products) to about 2^-16.  Error measure: max |C_tc - C_f64| / max |C_f64|
per bin, over the finished (Hermitian, scaled) CSM.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = {'tc_tf32': 2e-3, 'tc_bf16x3': 1e-4}


def _samples(S, M, dtype, seed):
    g = torch.Generator(device='cuda').manual_seed(seed)
    # a few coherent sources plus noise, so that the CSM has structure and a dominant diagonal
    t = torch.randn((S, 3), generator=g, device='cuda', dtype=torch.float64)
    mix = torch.randn((3, M), generator=g, device='cuda', dtype=torch.float64)
    x = t @ mix + 0.3 * torch.randn((S, M), generator=g, device='cuda', dtype=torch.float64)
    return x.to(dtype).contiguous()


@pytest.mark.parametrize('precision', ['tc_tf32', 'tc_bf16x3'])
@pytest.mark.parametrize('M,N,S,dtype', [(8, 128, 4000, torch.float64), (40, 256, 9000, torch.float32),
                                         (64, 1024, 51200, torch.float32), (130, 512, 20000, torch.float64),
                                         (256, 1024, 40000, torch.float32), (20, 4096, 40000, torch.float32),
                                         (9, 8192, 60000, torch.float64), (6, 16384, 70000, torch.float32)])
def test_tc_csm_vs_f64(precision, M, N, S, dtype):
    from acoular_b200 import device as D
    x = _samples(S, M, dtype, seed=M + N)
    ref = D.calc_csm(x, N, 'Hanning', '50%', 'complex128').cpu().numpy()
    got = D.calc_csm(x, N, 'Hanning', '50%', precision).cpu().numpy()
    assert got.shape == ref.shape and got.dtype == np.complex128
    scale = np.abs(ref).max(axis=(1, 2))
    err = np.abs(got - ref).max(axis=(1, 2)) / scale
    assert float(err.max()) <= TOL[precision], float(err.max())
    # Hermitian, real non-negative diagonal (as the finished CSM always is)
    assert np.allclose(got, np.conj(np.transpose(got, (0, 2, 1))), rtol=0, atol=1e-12 * scale.max())
    assert (np.real(np.diagonal(got, axis1=1, axis2=2)) >= 0).all()


@pytest.mark.parametrize('precision', ['tc_tf32', 'tc_bf16x3'])
def test_tc_csm_bin_range_and_chunks(precision):
    """A bin subset and a workspace that forces several window chunks give the same sums as one pass."""
    from acoular_b200 import device as D
    x = _samples(30000, 48, torch.float32, seed=3)
    whole = D.calc_csm(x, 512, 'Hanning', '50%', precision, bin_lo=40, num_bins=17).cpu().numpy()
    ref = D.calc_csm(x, 512, 'Hanning', '50%', 'complex128', bin_lo=40, num_bins=17).cpu().numpy()
    per32 = D.N.lib().acb_csm_workspace_bytes(48, 17, 32, D.CSM_PRECISIONS[precision])
    chunked = D.calc_csm(x, 512, 'Hanning', '50%', precision, bin_lo=40, num_bins=17,
                         max_workspace_bytes=2 * per32).cpu().numpy()
    scale = np.abs(ref).max()
    assert np.abs(whole - ref).max() / scale <= TOL[precision]
    assert np.abs(chunked - whole).max() / scale <= 1e-6


def test_tc_csm_then_tc_map_vs_oracle():
    """End to end: tensor-core CSM and tensor-core map against the FP64 CSM and FP64 map."""
    from acoular_b200 import device as D
    from acoular_b200.microphones import disk_mics
    from oracle import oracle as O
    M, N = 64, 256
    mpos = disk_mics(M, 0.5, seed=5).pos
    src = np.array([[0.1], [-0.05], [-0.5]])
    fs = 51200.0
    S = 25600
    rm = O.apparent_r(src, mpos).reshape(-1)
    g = torch.Generator(device='cuda').manual_seed(9)
    sig = torch.randn(S + 4096, generator=g, device='cuda', dtype=torch.float64)
    delay = torch.as_tensor(np.round(rm / 343.0 * fs).astype(np.int64), device='cuda')
    idx = torch.arange(S, device='cuda')[:, None] + 4096 - delay[None, :]
    x = (sig[idx] / torch.as_tensor(rm, device='cuda')[None, :]).to(torch.float32).contiguous()
    gx, gy = np.meshgrid(np.linspace(-0.3, 0.3, 31), np.linspace(-0.3, 0.3, 31), indexing='ij')
    gpos = np.vstack([gx.ravel(), gy.ravel(), np.full(gx.size, -0.5)])
    bins = torch.arange(20, 60, device='cuda')
    freqs = np.abs(np.fft.fftfreq(N, 1 / fs)[: N // 2 + 1])
    k = torch.as_tensor(2 * np.pi * freqs[20:60] / 343.0, device='cuda')
    mp, gp = torch.as_tensor(mpos, device='cuda'), torch.as_tensor(gpos, device='cuda')
    c64 = D.calc_csm(x, N, 'Hanning', '50%', 'complex128')[bins].contiguous()
    ref = D.map_f64(c64, k, mp, gp, 'true level', True, M / (M - 1.0)).cpu().numpy()
    ctc = D.calc_csm(x, N, 'Hanning', '50%', 'tc_tf32')[bins].contiguous()
    got = D.map_tc(ctc, k, mp, gp, 'true level', True, M / (M - 1.0), precision='tf32').cpu().numpy()
    err = np.abs(got - ref) / np.abs(ref).max(axis=1, keepdims=True)
    assert float(err.max()) <= 1e-3
    peak = ref.argmax(axis=1)
    lp = lambda v: 10 * np.log10(np.maximum(v / 4e-10, 1e-30))  # noqa: E731
    assert np.abs(lp(got[np.arange(len(peak)), peak]) - lp(ref[np.arange(len(peak)), peak])).max() <= 0.05
