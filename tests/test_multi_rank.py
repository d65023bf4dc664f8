"""The N > 1 host path of bench.py on CPU: two gloo ranks (one process each, as torchrun launches them)
set up the process group, meet at the barrier and agree on the max-over-ranks step time, which is what
the multi-GPU bench line reports.  No GPU and no data-path collective are involved: every rank runs an
independent replica of the single-GPU workload."""

import os
import socket
import sys
from pathlib import Path
from types import SimpleNamespace

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update({'RANK': str(rank), 'LOCAL_RANK': str(rank), 'WORLD_SIZE': str(world),
                       'MASTER_ADDR': '127.0.0.1', 'MASTER_PORT': str(port)})
    sys.path.insert(0, str(ROOT))
    import bench
    import torch.distributed as dist
    ws, r, local = bench.dist_setup(SimpleNamespace(impl='reference'))
    assert (ws, r, local) == (world, rank, rank)
    assert dist.get_backend() == 'gloo'
    bench.barrier(ws)
    # each rank's own step time; the bench reports the slowest rank's
    t = bench.max_over_ranks(10.0 + 5.0 * rank, ws)
    out[rank] = t
    bench.barrier(ws)
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_max_time():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        assert dict(out) == {0: 15.0, 1: 15.0}
