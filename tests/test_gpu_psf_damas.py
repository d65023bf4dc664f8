"""Point-spread functions (acb_psf_f64, PointSpreadFunction, fastFuncs.calcPointSpreadFunction) and
DAMAS (acb_damas_gauss_seidel_f64, BeamformerDamas, fastFuncs.damasSolverGaussSeidel) on the GPU,
against the reference's own results (tests/golden/psf_damas_kat.npz, produced by its numba kernels and
BeamformerDamas._calc) and the oracle.

Tolerances: PSF and maps <= 1e-10 of the largest value (the plain FP64 form's bar); float32-rounded
PSFs within one float32 ulp.  The Gauss-Seidel kernel sums each row in a different order than the
reference (column slices, then the solved block's updates), so solutions agree to rounding, <= 1e-10
of the largest value after 10-100 sweeps.
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

STEERS = ['classic', 'inverse', 'true level', 'true location']
TOL = 1e-10


def _rel(a, b):
    return float(np.abs(np.asarray(a) - b).max() / np.abs(b).max())


def _dev(a, dtype=None):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=dtype), device='cuda')


@pytest.fixture(scope='module')
def small(golden):
    s = golden('small_kat.npz')
    g = golden('psf_damas_kat.npz')
    r0, rm = O.apparent_r(s['gpos']), O.apparent_r(s['gpos'], s['mpos'])
    return s, g, r0, rm


@pytest.mark.parametrize('st', STEERS)
def test_psf_kernel_vs_reference(small, st):
    from acoular_b200 import device as D
    s, g, r0, rm = small
    G = rm.shape[0]
    k = 2 * np.pi * s['freqs0'][int(g['psf_bin'])] / 343.0
    key = st.replace(' ', '_')
    r0d, rmd = _dev(r0), _dev(rm)
    full = D.psf_f64(r0d, rmd, k, torch.arange(G, device='cuda'), st).cpu().numpy()
    assert _rel(full, g[f'psf_full_{key}']) <= TOL
    full32 = D.psf_f64(r0d, rmd, k, torch.arange(G, device='cuda'), st, round_f32=True).cpu().numpy()
    ref32 = g[f'psf_full32_{key}'].astype(np.float64)
    assert np.all(np.abs(full32 - ref32) <= 1.2e-7 * np.abs(ref32))
    assert np.array_equal(full32, full32.astype(np.float32).astype(np.float64))
    sel = D.psf_f64(r0d, rmd, k, _dev(g['src']), st, round_f32=True).cpu().numpy()
    ref = g[f'psf_src_{key}'].astype(np.float64)
    assert np.all(np.abs(sel - ref) <= 1.2e-7 * np.abs(ref))
    # uniform-flow distances, given as they are
    flow = D.psf_f64(_dev(g['flow_r0']), _dev(g['flow_rm']), k, _dev(g['src']), st).cpu().numpy()
    assert _rel(flow, g[f'psf_flow_{key}']) <= TOL
    # the oracle agrees on a larger set of wave numbers
    for kk in (0.5, 37.0, 180.0):
        got = D.psf_f64(r0d, rmd, kk, _dev(g['src']), st).cpu().numpy()
        assert _rel(got, O.psf(st, r0, rm, kk, g['src'])) <= TOL


@pytest.mark.parametrize('M', [45, 300])
@pytest.mark.parametrize('st', STEERS)
def test_psf_kernel_mic_counts(st, M):
    """Mic counts past one 32-mic group and not a multiple of 32 (45: a partial last group), and past one
    256-mic shared-memory chunk (300: a second chunk, itself partial), against the oracle at 1e-10."""
    from acoular_b200 import device as D
    rng = np.random.RandomState(M)
    mpos = np.vstack([rng.uniform(-0.6, 0.6, (2, M)), rng.uniform(-0.02, 0.02, (1, M))])
    g = np.linspace(-0.3, 0.3, 17)
    gx, gy = np.meshgrid(g, g, indexing='ij')
    gpos = np.vstack([gx.ravel(), gy.ravel(), np.full(gx.size, 0.8)])
    r0, rm = O.apparent_r(gpos), O.apparent_r(gpos, mpos)
    src = np.array([0, 50, 144, 288])
    for k in (3.0, 90.0):
        got = D.psf_f64(_dev(r0), _dev(rm), k, _dev(src), st).cpu().numpy()
        assert _rel(got, O.psf(st, r0, rm, k, src)) <= TOL


def test_psf_source_index_checks(small):
    """Host indices outside the grid raise; device indices outside it give NaN columns (no stray read)."""
    from acoular_b200 import device as D
    s, g, r0, rm = small
    r0d, rmd = _dev(r0), _dev(rm)
    with pytest.raises(IndexError):
        D.psf_f64(r0d, rmd, 10.0, np.array([0, 81]), 'classic')
    out = D.psf_f64(r0d, rmd, 10.0, torch.tensor([3, -1, 81, 40], device='cuda'), 'classic').cpu().numpy()
    assert np.isnan(out[:, 1]).all() and np.isnan(out[:, 2]).all()
    ref = O.psf('classic', r0, rm, 10.0, [3, 40])
    assert _rel(out[:, [0, 3]], ref) <= TOL


def test_psf_class_and_dropin(small):
    import acoular_b200 as ac
    from acoular_b200 import fastFuncs as F
    s, g, r0, rm = small
    f = float(s['freqs0'][int(g['psf_bin'])])
    mics, grid = ac.MicGeom(pos_total=s['mpos']), ac.ImportGrid(pos=s['gpos'])
    for st in STEERS:
        key = st.replace(' ', '_')
        steer = ac.SteeringVector(grid=grid, mics=mics, steer_type=st)
        p = ac.PointSpreadFunction(steer=steer, calcmode='full', freq=f)
        assert p.psf.shape == (81, 81) and p.psf.dtype == np.float64
        assert _rel(p.psf, g[f'psf_full_{key}']) <= TOL
        for mode in ('single', 'block', 'full', 'readonly'):
            q = ac.PointSpreadFunction(steer=steer, grid_indices=g['src'], calcmode=mode, precision='float32', freq=f)
            res = q.psf
            assert res.shape == (81, 3) and res.dtype == np.float32
            ref = g[f'psf_src_{key}']
            assert np.all(np.abs(res.astype(np.float64) - ref) <= 1.2e-7 * np.abs(ref))
        got = F.calcPointSpreadFunction(st, r0, rm, 2 * np.pi * f / 343.0, [3, 40, 77], 'float64')
        assert got.dtype == np.float64 and _rel(got, g[f'psf_full_{key}'][:, [3, 40, 77]]) <= TOL


def test_psf_custom_steering_matches_formulation(small):
    """A steering object other than SteeringVector takes |h^H a|^2; for the classic formulation's own
    vectors this equals the classic PSF."""
    import acoular_b200 as ac
    s, g, _, _ = small
    f = float(s['freqs0'][int(g['psf_bin'])])

    class MySteer(ac.SteeringVector):
        pass

    steer = MySteer(grid=ac.ImportGrid(pos=s['gpos']), mics=ac.MicGeom(pos_total=s['mpos']), steer_type='classic')
    got = ac.PointSpreadFunction(steer=steer, grid_indices=g['src'], calcmode='block', freq=f).psf
    h = steer.steer_vector(f)
    t = steer.transfer(f, g['src'])
    ref = np.abs(h.conj() @ t.T) ** 2
    assert _rel(got, ref) <= 1e-12


@pytest.mark.parametrize('cta', [0, 1, 2, 4, 8])
def test_damas_kernel_vs_oracle(small, cta):
    """Gauss-Seidel kernel on the reference's PSF and maps, every cluster size, against the oracle."""
    from acoular_b200 import device as D
    s, g, _, _ = small
    b = int(g['psf_bin']) - 10           # small_kat maps cover bins 10..30
    for st in STEERS:
        key = st.replace(' ', '_')
        A = g[f'psf_full_{key}']
        for rd in (False, True):
            y = np.maximum(s[f'map_{key}_{int(rd)}'][b], 0.0) if rd else s[f'map_{key}_{int(rd)}'][b]
            for n_iter, relax in ((10, 0.98), (100, 1.0), (3, 0.5)):
                x = D.damas_gauss_seidel(_dev(A[None]), _dev(y[None]), n_iter, relax, cta_per_bin=cta)
                ref = O.damas_gauss_seidel(A, y, n_iter, relax, y.copy())
                assert _rel(x.cpu().numpy()[0], ref) <= TOL, (st, rd, n_iter)


@pytest.mark.parametrize('G', [1, 5, 31, 32, 33, 64, 95, 200])
def test_damas_kernel_ragged_sizes(G):
    """Grids that are not multiples of the 32-row block (one block, a last block of one row, ...)."""
    from acoular_b200 import device as D
    rng = np.random.default_rng(G)
    B = 3
    A = rng.uniform(0.0, 1.0, (B, G, G)) / G
    A[:, np.arange(G), np.arange(G)] = 1.0
    y = rng.uniform(-0.2, 1.0, (B, G))
    x0 = rng.uniform(0.0, 1.0, (B, G))
    ref = O.damas_gauss_seidel(A, y, 7, 0.9, x0.copy())
    for cta in (1, 2, 8):
        x = D.damas_gauss_seidel(_dev(A), _dev(y), 7, 0.9, solution=_dev(x0), cta_per_bin=cta).cpu().numpy()
        assert _rel(x, ref) <= TOL, (G, cta)
        assert (x >= 0).all()


def test_damas_kernel_many_bins_and_zero_iterations():
    from acoular_b200 import device as D
    rng = np.random.default_rng(5)
    B, G = 300, 40                         # more bins than SMs: one CTA per bin
    A = rng.uniform(0.0, 1.0, (B, G, G)) / G
    A[:, np.arange(G), np.arange(G)] = 1.0
    y = rng.uniform(0.0, 1.0, (B, G))
    x = D.damas_gauss_seidel(_dev(A), _dev(y), 5, 1.0).cpu().numpy()
    assert _rel(x, O.damas_gauss_seidel(A, y, 5, 1.0, y.copy())) <= TOL
    x0 = rng.uniform(0.0, 1.0, (B, G))
    same = D.damas_gauss_seidel(_dev(A), _dev(y), 0, 1.0, solution=_dev(x0)).cpu().numpy()
    assert np.array_equal(same, x0)


def test_damas_kernel_errors():
    from acoular_b200 import device as D
    A = torch.zeros((1, 4, 4), dtype=torch.float64, device='cuda')
    y = torch.zeros((1, 4), dtype=torch.float64, device='cuda')
    with pytest.raises(RuntimeError):
        D.damas_gauss_seidel(A, y, 1, 1.0, cta_per_bin=3)
    with pytest.raises(ValueError):
        D.damas_gauss_seidel(A[:, :3], y, 1, 1.0)
    big = 40000                            # the solution does not fit a CTA's shared memory
    with pytest.raises(RuntimeError):
        D.damas_gauss_seidel(_FakeBig(big), torch.zeros((1, big), dtype=torch.float64, device='cuda'), 1, 1.0)


class _FakeBig:
    """Shape-only stand-in for a (1, G, G) PSF: the size check fails before any access."""

    def __init__(self, G):
        self.shape = (1, G, G)
        self.dtype = torch.float64

    def is_contiguous(self):
        return True

    def data_ptr(self):
        return 16


@pytest.mark.parametrize('st', STEERS)
def test_beamformer_damas_class_vs_reference(small, st):
    """TimeSamples -> PowerSpectra -> BeamformerDamas.result against BeamformerDamas._calc of the
    reference (n_iter 10, damp 0.98: its regression settings)."""
    import acoular_b200 as ac
    s, g, _, _ = small
    ts = ac.TimeSamples(data=s['data'], sample_freq=float(s['fs']))
    ps = ac.PowerSpectra(source=ts, block_size=128, window='Hanning', overlap='50%')
    steer = ac.SteeringVector(grid=ac.ImportGrid(pos=s['gpos']), mics=ac.MicGeom(pos_total=s['mpos']),
                              steer_type=st)
    key = st.replace(' ', '_')
    for rd in (False, True):
        bf = ac.BeamformerDamas(freq_data=ps, steer=steer, r_diag=rd, n_iter=10, damp=0.98)
        got = np.array([bf.result[int(i)] for i in g['bins']])
        assert _rel(got, g[f'damas_{key}_{int(rd)}']) <= 1e-9, rd
        assert (got >= 0).all()
    if st == 'classic':
        bf = ac.BeamformerDamas(freq_data=ps, steer=steer, r_diag=False)
        assert bf.n_iter == 100 and bf.damp == 1.0 and bf.calcmode == 'full'
        got = np.array([bf.result[int(i)] for i in g['bins']])
        assert _rel(got, g['damas_default_classic_0']) <= 1e-9
    if st == 'true level':
        bf = ac.BeamformerDamas(freq_data=ps, steer=steer, r_diag=True, n_iter=10, damp=0.98,
                                psf_precision='float32', psf_budget_bytes=1)
        got = np.array([bf.result[int(i)] for i in g['bins']])
        assert _rel(got, g['damas_f32_true_level_1']) <= 1e-9


def test_beamformer_damas_64mic_band(golden):
    """The 64-mic, 1681-point workload: two bins of the 8 kHz third-octave band, against the
    reference's BeamformerDamas (its own CSM, imported)."""
    import acoular_b200 as ac
    from acoular_b200 import workloads
    c1 = golden('config1_band.npz')
    g = golden('psf_damas_kat.npz')
    wl = workloads.three_sources_64()
    freqs = c1['freqs']
    csm = np.zeros((freqs.size, 64, 64), dtype=np.complex128)
    csm[c1['band_bins']] = c1['csm_band']
    ps = ac.PowerSpectraImport(csm=csm, frequencies=freqs)
    for st, rd in (('classic', False), ('true level', True)):
        steer = ac.SteeringVector(grid=wl.grid, mics=wl.mics, steer_type=st)
        bf = ac.BeamformerDamas(freq_data=ps, steer=steer, r_diag=rd, n_iter=10, damp=0.98)
        got = np.array([bf.result[int(i)] for i in g['c1_bins']])
        assert _rel(got, g[f'c1_damas_{st.replace(" ", "_")}_{int(rd)}']) <= 1e-9, st


def test_damas_dropin(small):
    from acoular_b200 import fastFuncs as F
    s, g, _, _ = small
    A = g['psf_full_classic']
    y = s['map_classic_0'][10]
    x = y.copy()
    out = F.damasSolverGaussSeidel(A, y, 10, 0.98, x)
    assert out is x
    assert _rel(x, O.damas_gauss_seidel(A, y, 10, 0.98, y.copy())) <= TOL
