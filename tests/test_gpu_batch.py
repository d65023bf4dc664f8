"""Batched uneven instances (CSM + map in one plan, optionally one CUDA graph)."""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _instances(n=6, seed=11):
    from acoular_b200.batch import Instance
    rng = np.random.RandomState(seed)
    out = []
    for i in range(n):
        M = int(rng.choice([8, 16, 33, 64]))
        N = int(rng.choice([128, 256, 512]))
        side = int(rng.randint(5, 30))
        mpos = np.vstack([rng.uniform(-0.5, 0.5, (2, M)), np.zeros((1, M))])
        g = np.linspace(-0.4, 0.4, side)
        gx, gy = np.meshgrid(g, g, indexing='ij')
        gpos = np.vstack([gx.ravel(), gy.ravel(), np.full(side * side, -0.6 - 0.1 * i)])
        S = N * 6 + int(rng.randint(0, N))
        data = rng.randn(S, M).astype(np.float32)
        F = N // 2 + 1
        nb = int(rng.randint(1, 8))
        b0 = int(rng.randint(1, F - nb))
        out.append(Instance(samples=data, mpos=mpos, gpos=gpos, sample_freq=51200.0, block_size=N, bin_lo=b0,
                            num_bins=nb, precision=str(rng.choice(['complex64', 'complex128']))))
    return out


@pytest.mark.parametrize('form', ['tc', 'f64'])
def test_batch_plan_equals_instances_alone(form):
    from acoular_b200 import device as D
    from acoular_b200.batch import BatchPlan
    insts = _instances()
    plan = BatchPlan(insts, form=form)
    outs = [o.cpu().numpy() for o in plan.run()]
    dev = plan.dev
    for it, got in zip(insts, outs):
        M = it.mpos.shape[1]
        x = torch.as_tensor(it.samples, device=dev)
        csm = D.calc_csm(x, it.block_size, it.window, it.overlap, it.precision, bin_lo=it.bin_lo, num_bins=it.num_bins)
        freqs = O.fftfreq(it.block_size, it.sample_freq)[it.bin_lo:it.bin_lo + it.num_bins]
        k = torch.as_tensor(2 * np.pi * freqs / 343.0, device=dev)
        fn = D.map_tc if form == 'tc' else D.map_f64
        alone = fn(csm, k, torch.as_tensor(it.mpos, device=dev), torch.as_tensor(it.gpos, device=dev), it.steer_type,
                   True, M / (M - 1.0)).cpu().numpy()
        assert np.array_equal(got, alone)
        # and against the oracle (CSM of the float32 samples, all bins, then the instance's band)
        csm_ref = O.calc_csm(it.samples.astype(np.float64), it.block_size, it.window, it.overlap, it.precision)
        bins = np.arange(it.bin_lo, it.bin_lo + it.num_bins)
        ref = O.beamformer_calc(csm_ref, O.fftfreq(it.block_size, it.sample_freq), bins, O.apparent_r(it.gpos),
                                O.apparent_r(it.gpos, it.mpos), 343.0, it.steer_type, True)[bins]
        tol = 1e-3 if form == 'tc' else (1e-10 if it.precision == 'complex128' else 1e-5)
        assert np.abs(got - ref).max() <= tol * np.abs(ref).max()


def test_batch_plan_graph_replay_with_new_data():
    from acoular_b200.batch import BatchPlan
    insts = _instances(seed=23)
    plan = BatchPlan(insts).capture()
    first = [o.clone() for o in plan.run()]
    rng = np.random.RandomState(1)
    new = [rng.randn(*it.samples.shape).astype(np.float32) for it in insts]
    plan.load_samples(new)
    second = [o.clone() for o in plan.run()]
    eager = BatchPlan([type(it)(**{**it.__dict__, 'samples': x}) for it, x in zip(insts, new)])
    third = eager.run()
    for a, b, c in zip(first, second, third):
        assert not torch.equal(a, b)
        assert torch.equal(b, c)
