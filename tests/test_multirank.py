"""Multi-rank host logic on CPU (gloo, world size 2): molecules sharded
over the ranks by size, each rank computing its shard, rank 0 gathering the
lists in the original order.  The per-rank computation here is the oracle
(the GPU is not needed to test the distribution of work)."""
import os
import socket

import numpy as np
import pytest

from conftest import ROOT


def test_shard_molecules_balances_and_covers(pac):
    sizes = pac.batch_sizes(300)
    for world in (1, 2, 3, 8):
        parts = pac.shard_molecules(sizes, world)
        allm = np.sort(np.concatenate(parts))
        np.testing.assert_array_equal(allm, np.arange(len(sizes)))
        loads = [int(sizes[p].sum()) for p in parts]
        # greedy largest-first: no rank exceeds the mean by more than one molecule
        assert max(loads) - sum(loads) / world <= sizes.max()


def _worker(rank, world, port, out_path):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import __graft_entry__ as ge
    pac, orc = ge.load_package(), ge.load_oracle()
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world)
    try:
        sizes = np.array([220, 900, 310, 640, 450])
        balls, off = pac.batch(sizes, seed=pac.SEED_BASE + 90)

        def run(b, o):
            return [orc.alpha_complex(b[o[m]:o[m + 1]], 1.4, 0.5)[:3] for m in range(len(o) - 1)]
        res = pac.sharded_batch(balls, off, rank, world, run)
        if rank == 0:
            np.savez(out_path, **{"%d_%d" % (m, k): a for m, r in enumerate(res)
                                  for k, a in enumerate(r)})
        else:
            assert res is None
    finally:
        dist.destroy_process_group()


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_batch_two_ranks_gloo(pac, orc, tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "gathered.npz")
    mp.start_processes(_worker, args=(2, _port(), out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    sizes = np.array([220, 900, 310, 640, 450])
    balls, off = pac.batch(sizes, seed=pac.SEED_BASE + 90)
    for m in range(len(sizes)):
        want = orc.alpha_complex(balls[off[m]:off[m + 1]], 1.4, 0.5)[:3]
        for k in range(3):
            np.testing.assert_array_equal(got["%d_%d" % (m, k)], want[k])
