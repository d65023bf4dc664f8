"""Eigenvalue beamformers on the GPU (acb_map_eig_f64, BeamformerEig, BeamformerMusic) against the
reference's own results (tests/golden/eig_kat.npz, produced by its numba kernel and LAPACK eigh).

Kernel parity uses the reference's eigen-decomposition as input: <= 1e-10 of the max per bin, the
plain form's bar.  End to end (device eigh) is checked on the well-separated largest component only:
in these noise-free fixtures the small eigenvalues are round-off, so their eigenvectors (and any map
built from them alone) are not determined by the CSM.
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

STEERS = ['classic', 'inverse', 'true level', 'true location']
TOL = 1e-10


def _rel(a, b):
    return float((np.abs(a - b).max(axis=-1) / np.abs(b).max(axis=-1)).max())


def _dev(a):
    return torch.as_tensor(np.ascontiguousarray(a), device='cuda')


@pytest.mark.parametrize('tag', ['s', 'c1'])
def test_map_eig_kernel_vs_reference(golden, tag):
    from acoular_b200 import device as D
    g = golden('eig_kat.npz')
    mpos, gpos, freqs = g[f'{tag}_mpos'], g[f'{tag}_gpos'], g[f'{tag}_freqs']
    eva, eve = g[f'{tag}_eigvals'], g[f'{tag}_eigvecs']
    M = mpos.shape[1]
    k = _dev(2 * np.pi * freqs / 343.0)
    mp, gp = _dev(mpos), _dev(gpos)
    for n in (-1, 0, M // 2):
        na = O.eig_na(n, M)
        lam, vec = _dev(eva[:, na:na + 1]), _dev(eve[:, :, na:na + 1])
        for st in STEERS:
            for rd in (False, True):
                ref = g[f'{tag}_eig_n{n}_{st.replace(" ", "_")}_{int(rd)}']
                out = D.map_eig_f64(lam, vec, k, mp, gp, st, rd, O.sig_loss_norm(rd, M), clip_negative=rd)
                assert _rel(out.cpu().numpy(), ref) <= TOL, (n, st, rd)
    for n in (1, 3):
        ne = M - O.eig_na(n, M)
        lam, vec = _dev(eva[:, :ne]), _dev(eve[:, :, :ne])
        for st in STEERS:
            ref = g[f'{tag}_music_n{n}_{st.replace(" ", "_")}']
            b = D.map_eig_f64(lam, vec, k, mp, gp, st, False, float(M) ** 2, clip_negative=False)
            got = (4e-10 * b.min(dim=1, keepdim=True).values / b).cpu().numpy()
            assert _rel(got, ref) <= TOL, (n, st)


def test_beamformerfreq_eig_dropin(golden):
    """fastFuncs.beamformerFreq with an eigen tuple, as BeamformerEig._calc calls it."""
    from acoular_b200 import fastFuncs as F
    g = golden('eig_kat.npz')
    mpos, gpos, freqs = g['s_mpos'], g['s_gpos'], g['s_freqs']
    eva, eve = g['s_eigvals'], g['s_eigvecs']
    r0, rm = O.apparent_r(gpos), O.apparent_r(gpos, mpos)
    for st in STEERS:
        for rd in (False, True):
            for b in (0, 7):
                k = 2 * np.pi * freqs[b] / 343.0
                lam, vec = np.array(eva[b, -2:]), np.ascontiguousarray(eve[b][:, -2:])
                got, gn = F.beamformerFreq(st, rd, 1.25, (r0, rm, k), (lam, vec))
                ref, rn = O.beamformer_freq_eig(st, rd, 1.25, r0, rm, k, lam, vec)
                assert np.abs(got - ref).max() <= TOL * np.abs(ref).max()
                assert np.abs(gn - rn).max() <= TOL * np.abs(rn).max()


def test_beamformer_eig_class_end_to_end(golden):
    """TimeSamples -> PowerSpectra (device CSM + device eigh) -> BeamformerEig.result, largest component."""
    import acoular_b200 as ac
    s = golden('small_kat.npz')
    g = golden('eig_kat.npz')
    ts = ac.TimeSamples(data=s['data'], sample_freq=float(s['fs']))
    ps = ac.PowerSpectra(source=ts, block_size=128, window='Hanning', overlap='50%')
    mics = ac.MicGeom(pos_total=s['mpos'])
    grid = ac.ImportGrid(pos=s['gpos'])
    bins = g['s_bins']
    for st in STEERS:
        for rd in (False, True):
            bf = ac.BeamformerEig(freq_data=ps, steer=ac.SteeringVector(grid=grid, mics=mics, steer_type=st),
                                  r_diag=rd, n=-1)
            got = np.array(bf.result[bins[0]:bins[-1] + 1])
            ref = g[f's_eig_n-1_{st.replace(" ", "_")}_{int(rd)}']
            assert _rel(got, ref) <= 1e-8, (st, rd)
    mu = ac.BeamformerMusic(freq_data=ps, steer=ac.SteeringVector(grid=grid, mics=mics), n=3)
    assert mu.na == 3 and mu.r_diag is False
    res = np.array(mu.result[bins[0]:bins[-1] + 1])
    assert np.isfinite(res).all() and (res > 0).all()


@pytest.mark.parametrize('M', [1, 2, 5, 8, 33, 64, 256, 300])
def test_heevd_against_lapack(M):
    """acb_heevd_f64 (Householder tridiagonalisation, implicit QL, back-transformation) on CSM-like matrices:
    eigenvalues ascending within 1e-12 of numpy's (relative to the largest), residual |A V - V diag(w)| and
    |V^H V - I| within 1e-12; a zero, an identity and a rank-1 matrix among them."""
    from acoular_b200 import device as D
    rng = np.random.RandomState(M)
    mats = []
    for _ in range(3):
        X = rng.randn(2 * M, M) + 1j * rng.randn(2 * M, M)
        A = X.conj().T @ X / (2 * M)
        a = np.exp(-1j * rng.uniform(0, 6, M)) / rng.uniform(0.5, 2.0, M)
        mats.append(A + 40.0 * np.outer(a, a.conj()))
    a = np.exp(1j * rng.uniform(0, 6, M))
    mats += [np.zeros((M, M), complex), np.eye(M, dtype=complex), np.outer(a, a.conj())]
    C = np.stack(mats)
    w, V, info = D.heevd_f64(_dev(C))
    w, V = w.cpu().numpy(), V.cpu().numpy()
    assert not int(info.max())
    for A, wb, Vb in zip(C, w, V):
        wr = np.linalg.eigvalsh(A)
        scale = max(np.abs(wr).max(), 1e-300)
        assert np.all(np.diff(wb) >= 0)
        assert np.abs(wb - wr).max() <= 1e-12 * scale
        assert np.abs(A @ Vb - Vb * wb).max() <= 1e-12 * max(scale, 1.0)
        assert np.abs(Vb.conj().T @ Vb - np.eye(M)).max() <= 1e-12


def test_power_spectra_evd_device_matches_host(golden):
    """PowerSpectra.evd_device (the device eigendecomposition) against the host LAPACK one of the same CSM:
    eigenvalues within 1e-12 of max, and a well-separated largest component's eigenvector up to its phase."""
    import acoular_b200 as ac
    s = golden('small_kat.npz')
    ps = ac.PowerSpectra(source=ac.TimeSamples(data=s['data'], sample_freq=float(s['fs'])), block_size=128,
                         window='Hanning', overlap='50%')
    ev, evec = ps.evd_device
    ev, evec = ev.cpu().numpy(), evec.cpu().numpy()
    wr, vr = ps.eigvals, ps.eigvecs
    for b in range(ev.shape[0]):
        assert np.abs(ev[b] - wr[b]).max() <= 1e-12 * max(np.abs(wr[b]).max(), 1e-300)
        if wr[b, -1] > 1e3 * max(wr[b, -2], 1e-300):
            ph = np.vdot(vr[b][:, -1], evec[b][:, -1])
            assert abs(abs(ph) - 1.0) <= 1e-9


@pytest.mark.parametrize('M', [1, 2, 5, 8, 33, 64, 256, 300])
def test_heevd_select_against_lapack(M):
    """acb_heevd_select_f64 (multisection on Sturm counts, inverse iteration, back-transformation) on the same
    CSM-like matrices: the selected eigenvalues within 1e-12 of numpy's (relative to the largest); each selected
    vector of unit norm with residual |A v - w v| within 1e-11 of the largest eigenvalue, and, where the
    eigenvalue is separated from its neighbours by 1e-6 of the largest, equal to numpy's up to a phase."""
    from acoular_b200 import device as D
    rng = np.random.RandomState(M + 7)
    mats = []
    for _ in range(3):
        X = rng.randn(2 * M, M) + 1j * rng.randn(2 * M, M)
        A = X.conj().T @ X / (2 * M)
        a = np.exp(-1j * rng.uniform(0, 6, M)) / rng.uniform(0.5, 2.0, M)
        mats.append(A + 40.0 * np.outer(a, a.conj()))
    a = np.exp(1j * rng.uniform(0, 6, M))
    mats += [np.zeros((M, M), complex), np.eye(M, dtype=complex), np.outer(a, a.conj())]
    C = np.stack(mats)
    for ranks in ([M - 1], [0], sorted({0, M // 2, M - 1})):
        w, V = D.heevd_select_f64(_dev(C), ranks)
        w, V = w.cpu().numpy(), V.cpu().numpy()
        for A, wb, Vb in zip(C, w, V):
            wr, vr = np.linalg.eigh(A)
            scale = max(np.abs(wr).max(), 1e-300)
            for j, r in enumerate(ranks):
                assert abs(wb[j] - wr[r]) <= 1e-12 * scale
                v = Vb[:, j]
                assert abs(np.linalg.norm(v) - 1.0) <= 1e-12
                assert np.abs(A @ v - wb[j] * v).max() <= 1e-11 * max(scale, 1.0)
                gap = min([abs(wr[r] - wr[q]) for q in (r - 1, r + 1) if 0 <= q < M] or [scale])
                if gap > 1e-6 * scale:
                    assert abs(abs(np.vdot(vr[:, r], v)) - 1.0) <= 1e-9


def test_beamformer_eig_selected_path_matches_full(golden):
    """BeamformerEig n = -1 through the selected-eigenpair solver and through a cached full decomposition
    (PowerSpectra.evd_device) give the same map to 1e-9 of max on the small fixture's well-separated bins."""
    import acoular_b200 as ac
    s = golden('small_kat.npz')
    g = golden('eig_kat.npz')
    ps = ac.PowerSpectra(source=ac.TimeSamples(data=s['data'], sample_freq=float(s['fs'])), block_size=128,
                         window='Hanning', overlap='50%')
    mics = ac.MicGeom(pos_total=s['mpos'])
    grid = ac.ImportGrid(pos=s['gpos'])
    st = ac.SteeringVector(grid=grid, mics=mics)
    bins = np.asarray(g['s_bins'])
    sel = np.array(ac.BeamformerEig(freq_data=ps, steer=st, n=-1).result[bins[0]:bins[-1] + 1])
    ps.evd_device   # cache the full decomposition: the same class now takes its columns
    full = np.array(ac.BeamformerEig(freq_data=ps, steer=st, n=-1).result[bins[0]:bins[-1] + 1])
    wr = ps.eigvals
    for j, b in enumerate(bins):
        if wr[b, -1] > 1e3 * max(wr[b, -2], 1e-300):
            assert np.abs(sel[j] - full[j]).max() <= 1e-9 * max(np.abs(full[j]).max(), 1e-300)
