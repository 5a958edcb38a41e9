"""bench.py's multi-rank plumbing on CPU: two gloo ranks (no GPU).

Under torchrun each rank runs its own replica of the workload (its own seed,
no data-path collective); timings are reduced with a max over ranks and the
whole-job rate is ranks x units / that time.  The reference arm runs on rank 0
only; the other ranks exit 0 without work.
"""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(ws), "LOCAL_RANK": str(rank)})
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        got_ws, got_rank, _ = bench.dist_env()
        # per-rank timings (ms) and a rate
        mx = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 3.0], got_ws, device="cpu")
        rate = bench.job_rate(1000, got_ws, mx[0] * 1e-3)
        # reference arm: rank 1 returns at once and prints nothing
        out = ""
        if rank != 0:
            buf = io.StringIO()
            with redirect_stdout(buf):
                rc = bench.reference_arm(type("A", (), {"steps": 1, "warmup": 0, "gpus": ws})())
            out = buf.getvalue()
        else:
            rc = 0
        q.put((rank, got_ws, got_rank, mx, rate, rc, out))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(ws):
        r = q.get(timeout=120)
        res[r[0]] = r
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in range(ws):
        _, got_ws, got_rank, mx, rate, rc, out = res[rank]
        assert got_ws == ws and got_rank == rank
        assert mx == [2.0, 10.0, 3.0]          # max over the two ranks, element-wise
        assert rate == pytest.approx(ws * 1000 / 2e-3)
        assert rc == 0
    assert res[1][6] == ""                      # rank 1 of the reference arm prints nothing


def test_replicas_have_own_seeds():
    sys.path.insert(0, ROOT)
    import bench
    a = bench.make_points(0)
    b = bench.make_points(1)
    assert a[0].shape == b[0].shape == (bench.N_POINTS, 3)
    assert not np.array_equal(a[0], b[0])
    assert np.all(a[0] >= 0) and np.all(a[0] < 1)
