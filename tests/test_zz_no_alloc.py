"""The allocation-free tensor-core map entry point (acb_map_tc_noalloc) through the C ABI.

It serves callers that cannot allocate device memory when they call (a real-time acquisition loop
that must not risk cudaMalloc's device synchronisation, or a host program without a device
allocator): its scratch is a fixed 32 MiB array the library keeps on each GPU.  This file is
collected last so that a run stopping at the first failure has run every other test first.
"""

import ctypes

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu



def _inputs(M, G, nb, seed):
    rng = np.random.RandomState(seed)
    mpos = np.vstack([rng.uniform(-0.5, 0.5, (2, M)), np.zeros((1, M))])
    gpos = np.vstack([rng.uniform(-0.4, 0.4, (2, G)), np.full((1, G), -0.7)])
    X = rng.randn(nb, 2 * M, M) + 1j * rng.randn(nb, 2 * M, M)
    csm = np.einsum('fkm,fkn->fmn', X.conj(), X) / (2 * M)
    k = 2 * np.pi * np.linspace(800.0, 12000.0, nb) / 343.0
    return mpos, gpos, csm, k


def test_noalloc_matches_workspace_entry_point_on_two_calls():
    from acoular_b200 import _native as N
    from acoular_b200 import device as D
    dev = torch.device('cuda')
    L = N.lib()
    for M, G, nb in ((64, 3000, 5), (256, 1500, 4)):
        mpos, gpos, csm, k = _inputs(M, G, nb, seed=M + nb)
        c, kk = torch.as_tensor(csm, device=dev), torch.as_tensor(k, device=dev)
        mp, gp = torch.as_tensor(mpos, device=dev), torch.as_tensor(gpos, device=dev)
        p = D.map_params(M, G, nb, 'true level', True, O.sig_loss_norm(True, M))
        ws = torch.empty(L.acb_map_tc_workspace_bytes(M, nb, 0), dtype=torch.uint8, device=dev)
        ref = torch.empty((nb, G), dtype=torch.float64, device=dev)
        st = N.stream_handle()
        N.check(L.acb_map_tc(ctypes.byref(p), 0, c.data_ptr(), kk.data_ptr(), mp.data_ptr(), gp.data_ptr(),
                             ref.data_ptr(), None, ws.data_ptr(), ws.numel(), None, st), 'acb_map_tc')
        for _ in range(2):  # the shared array keeps the previous call's contents
            out = torch.full((nb, G), np.nan, dtype=torch.float64, device=dev)
            N.check(L.acb_map_tc_noalloc(ctypes.byref(p), 0, c.data_ptr(), kk.data_ptr(), mp.data_ptr(),
                                         gp.data_ptr(), out.data_ptr(), None, None, st), 'acb_map_tc_noalloc')
            torch.cuda.synchronize()
            a, b = out.cpu().numpy(), ref.cpu().numpy()
            assert np.isfinite(a).all()
            # the same kernel on the same inputs, only the scratch memory differs: bit for bit
            assert np.array_equal(a, b)


def test_noalloc_rejects_requests_beyond_its_array():
    from acoular_b200 import _native as N
    from acoular_b200 import device as D
    L = N.lib()
    M, nb = 256, 100  # 100 bins x 544 KB > 32 MiB
    assert L.acb_map_tc_workspace_bytes(M, nb, 0) > 32 << 20
    p = D.map_params(M, 1000, nb, 'classic', True, 1.0)
    assert L.acb_map_tc_noalloc(ctypes.byref(p), 0, 1, 1, 1, 1, 1, None, None, None) == 1  # ACB_ERR_SHAPE
