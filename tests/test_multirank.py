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


def slab_expectation(pac, orc, balls, sol, alpha, world):
    """Each rank's share of the restatement's complex under the slab
    partition (pac.slab_cuts): the simplices whose smallest vertex in cell
    order lies in the rank's range, in reference order."""
    E, T, Q, _ = orc.alpha_complex(balls, sol, alpha, orc.UPSTREAM, tet_ortho=True)
    order, cuts = pac.slab_cuts(balls, sol, alpha, world)
    pos = np.empty(len(balls), np.int64)
    pos[order] = np.arange(len(balls))
    parts = []
    for L in (E, T, Q):
        owner = pos[L.astype(np.int64)].min(1) if len(L) else np.zeros(0, np.int64)
        rank = np.searchsorted(cuts, owner, side="right") - 1
        parts.append([L[rank == r] for r in range(world)])
    return (E, T, Q), [tuple(parts[k][r] for k in range(3)) for r in range(world)]


def _slab_worker(rank, world, port, out_path):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import __graft_entry__ as ge
    pac, orc = ge.load_package(), ge.load_oracle()
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world)
    try:
        balls = pac.assembly(nx=2, ny=2, nz=1, per=1500)
        _, shares = slab_expectation(pac, orc, balls, 1.4, 1.0, world)
        got = pac._gather_rows(list(shares[rank]), rank, world)
        if rank == 0:
            np.savez(out_path, **{"%d_%d" % (r, k): got[r][k] for r in range(world)
                                  for k in range(3)})
        else:
            assert got is None
    finally:
        dist.destroy_process_group()


def test_slab_partition_two_ranks_gloo(pac, orc, tmp_path):
    """One assembly over two gloo ranks by cell-order slabs: each rank's
    share (here the restatement's simplices owned by the rank's slab,
    standing in for the GPU engine's slab pass) gathered on rank 0 in rank
    order is the whole complex, in the reference's order."""
    import torch.multiprocessing as mp
    out = str(tmp_path / "slabs.npz")
    world = 2
    mp.start_processes(_slab_worker, args=(world, _port(), out), nprocs=world, join=True,
                       start_method="spawn")
    got = np.load(out)
    balls = pac.assembly(nx=2, ny=2, nz=1, per=1500)
    full, shares = slab_expectation(pac, orc, balls, 1.4, 1.0, world)
    for k in range(3):
        cat = np.concatenate([got["%d_%d" % (r, k)] for r in range(world)])
        np.testing.assert_array_equal(cat, full[k])
        assert all(len(got["%d_%d" % (r, k)]) > 0 for r in range(world))


def test_slab_cuts_follow_cells(pac):
    balls = pac.assembly(nx=2, ny=2, nz=1, per=1500)
    for world in (1, 2, 3, 8):
        order, cuts = pac.slab_cuts(balls, 1.4, 1.0, world)
        assert cuts[0] == 0 and cuts[-1] == len(balls) and np.all(np.diff(cuts) >= 0)
        assert sorted(order.tolist()) == list(range(len(balls)))
