"""The bounded device-side waits of the tensor-core map: a wait that runs out ends the launch cleanly.

Every mbarrier wait of map_tc_kernel gives up after a limit (acb_tc_set_wait_limit_ns, 0.5 s by
default), raises the launch's error word, lets the CTA's own bulk copies and MMAs finish, frees its
tensor memory and returns.  Here the limit is set to 100 ns, far shorter than the bulk copies, steering
synthesis and MMAs that the pipeline's waits cover, so waits run out on a normal input (no fault, no trap, nothing that
never finishes); the test checks that the error word reports it, that the context stays usable, and
that the next launch at the default limit, which must allocate the tensor memory again, gives the
oracle's map with a clear error word.
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_tc_wait_timeout_reports_and_recovers():
    from acoular_b200 import _native as N
    from acoular_b200 import device as D
    dev = torch.device('cuda')
    L = N.lib()
    M, G, nb = 256, 40000, 4
    rng = np.random.RandomState(5)
    mpos = np.vstack([rng.uniform(-0.5, 0.5, (2, M)), np.zeros((1, M))])
    gpos = np.vstack([rng.uniform(-0.4, 0.4, (2, G)), np.full((1, G), -0.7)])
    X = rng.randn(nb, 2 * M, M) + 1j * rng.randn(nb, 2 * M, M)
    csm = np.einsum('fkm,fkn->fmn', X.conj(), X) / (2 * M)
    freqs = np.linspace(1000.0, 9000.0, nb)
    c, k = torch.as_tensor(csm, device=dev), torch.as_tensor(2 * np.pi * freqs / 343.0, device=dev)
    mp, gp = torch.as_tensor(mpos, device=dev), torch.as_tensor(gpos, device=dev)
    norm = O.sig_loss_norm(True, M)
    err = torch.zeros(1, dtype=torch.int32, device=dev)

    def run():
        err.zero_()
        out = D.map_tc(c, k, mp, gp, 'true level', True, norm, clip_negative=True, precision='tf32', error_word=err,
                       tuning=None)
        torch.cuda.synchronize()
        return out, int(err.item())

    run()                                         # at the default limit: no timeout
    assert int(err.item()) == 0
    prev = L.acb_tc_set_wait_limit_ns(100)
    try:
        flags = [run()[1] for _ in range(3)]
    finally:
        L.acb_tc_set_wait_limit_ns(prev)
    assert any(flags), flags                      # the short waits ran out and were reported
    out, flag = run()                             # the device is usable and the tensor memory was freed
    assert flag == 0
    r0, rm = O.apparent_r(gpos), O.apparent_r(gpos, mpos)
    ref = O.beamformer_calc(csm, freqs, range(nb), r0, rm, 343.0, 'true level', True)
    got = out.cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-3 * np.abs(ref).max()
