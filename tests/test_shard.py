"""Sharding of one problem across GPUs (Stk3DFMM_set_shard), host side: the
cost-balanced (LPT) assignment of work items, alone and as seen from two gloo
ranks.  The GPU side (sum over shards == unsharded result) is in
tests/test_gpu_shard.py."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def lpt(cost, nparts):
    from stkfmm_b200._lib import P_d, P_i, lib
    cost = np.ascontiguousarray(cost, dtype=np.float64)
    owner = np.zeros(len(cost), dtype=np.int32)
    rc = lib().stk_partition_lpt(len(cost), cost.ctypes.data_as(P_d), nparts, owner.ctypes.data_as(P_i))
    assert rc == 0
    return owner


def test_lpt_balance_and_determinism():
    rng = np.random.default_rng(0)
    cost = np.sort(rng.pareto(1.5, 5000) + 1.0)[::-1]
    for nparts in (1, 2, 3, 8):
        own = lpt(cost, nparts)
        assert own.min() >= 0 and own.max() < nparts
        load = np.bincount(own, weights=cost, minlength=nparts)
        # LPT: no part exceeds the lightest by more than one item
        assert load.max() - load.min() <= cost.max() + 1e-9
        assert np.array_equal(own, lpt(cost, nparts))
    assert np.all(lpt(cost, 1) == 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from test_shard import lpt
        cost = np.sort(np.random.default_rng(1).random(999) + 0.1)[::-1]   # same list on every rank
        mine = np.flatnonzero(lpt(cost, ws) == rank)
        n = torch.tensor([len(mine)])
        sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(ws)]
        dist.all_gather(sizes, n)
        buf = torch.full((int(max(s.item() for s in sizes)),), -1, dtype=torch.int64)
        buf[:len(mine)] = torch.as_tensor(mine)
        got = [torch.zeros_like(buf) for _ in range(ws)]
        dist.all_gather(got, buf)
        allidx = np.concatenate([g.numpy()[g.numpy() >= 0] for g in got])
        q.put((rank, sorted(allidx.tolist()) == list(range(len(cost))), len(allidx) == len(cost)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_cover_every_item_once():
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in range(ws)]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(r[1] and r[2] for r in res)


def test_far_owners_cover_every_node():
    """The M2L / S2L owners of a split far field: every node one rank, complete levels
    by parity type, loads balanced."""
    import stkfmm_b200 as S
    rng = np.random.default_rng(3)
    pts = rng.random((20000, 3))
    t = S.Octree(pts, 40, 0, sl=pts, trg=pts)
    off, _ = t.list("V")
    for nranks in (1, 2, 3, 4, 8):
        own = t.far_owners(nranks)
        assert own.min() >= 0 and own.max() < nranks
        cost = 1.0 + np.diff(off)
        load = np.bincount(own, weights=cost, minlength=nranks)
        assert load.max() <= 1.3 * load.mean() + cost.max()
    own = t.far_owners(8)
    for l in range(1, t.depth + 1):
        lev = np.flatnonzero(t.level == l)
        if len(lev) == 8 ** l:  # complete level: the owner is the parity type
            c = (t.ixyz[lev, 0] & 1) | (t.ixyz[lev, 1] & 1) << 1 | (t.ixyz[lev, 2] & 1) << 2
            assert np.array_equal(own[lev], c % 8)


def _split_rank(rank, ws, port, q):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import stkfmm_b200 as S
        # the same tree on every rank; each rank fills the downward densities of the nodes it
        # owns (here a per-node vector), one sum over the group gives every rank all of them
        rng = np.random.default_rng(5)
        pts = rng.random((8000, 3))
        t = S.Octree(pts, 40, 0, sl=pts, trg=pts)
        own = t.far_owners(ws)
        full = np.random.default_rng(6).normal(size=(t.num_nodes, 7))
        mine = np.where((own == rank)[:, None], full, 0.0)
        buf = torch.as_tensor(mine.copy())
        dist.all_reduce(buf, op=dist.ReduceOp.SUM)
        q.put((rank, float(np.abs(buf.numpy() - full).max())))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_far_field_reduction():
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_split_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in range(ws)]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(r[1] == 0.0 for r in res)
