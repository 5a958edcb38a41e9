"""GPU: one problem evaluated in shards (Stk3DFMM_set_shard).  Every shard is
run here in turn on the one GPU; the sum of the shards' outputs must equal the
unsharded evaluation (near field and full FMM)."""
import numpy as np
import pytest

from conftest import rel_l2
from helpers import clustered_points

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def case(n=6000, seed=2):
    rng = np.random.default_rng(seed)
    pts = np.minimum(clustered_points(rng, n, nclusters=5, sigma=0.05), 0.999)
    q = rng.uniform(-0.5, 0.5, (n, 1))
    d = rng.normal(size=(n, 3))
    return pts, q, d


def run(pts, q, d, shard, fmm_eval, prec=0):
    import stkfmm_b200 as S
    f = S.Stk3DFMM(8, 50, 0, 1, precision=prec)
    f.set_box(np.zeros(3), 1.0)
    f.set_points(pts, pts, pts)
    if shard is not None:
        f.set_shard(*shard)
    f.setup_tree(1)
    out = np.zeros((len(pts), 4))
    (f.evaluate_fmm if fmm_eval else f.evaluate_near)(1, q, out, d)
    return out, f.tree_stats(1)


@pytest.mark.parametrize("fmm_eval", [False, True])
@pytest.mark.parametrize("nranks", [2, 3])
def test_shards_sum_to_whole(torch_cuda, fmm_eval, nranks):
    pts, q, d = case()
    whole, st = run(pts, q, d, None, fmm_eval)
    parts = [run(pts, q, d, (r, nranks), fmm_eval) for r in range(nranks)]
    total = sum(p[0] for p in parts)
    assert rel_l2(total, whole) < 1e-14
    # the near-field pairs are split, not duplicated
    assert sum(p[1]["u_pairs_sl"] for p in parts) == st["u_pairs_sl"]
    assert all(p[1]["u_pairs_sl"] > 0 for p in parts)


def test_bad_shard_rejected(torch_cuda):
    import stkfmm_b200 as S
    f = S.Stk3DFMM(8, 50, 0, 1)
    for bad in ((2, 2), (-1, 2), (0, 0)):
        with pytest.raises(S.StkError):
            f.set_shard(*bad)


class HostGroup:
    """A shard group of host threads on one GPU: the collective copies each rank's
    device buffer to the host, sums the ranks' copies behind a barrier and writes
    the sum back.  Ranks meet on the host only -- no GPU work waits on another rank."""

    def __init__(self, n):
        import threading
        self.n = n
        self.bar = threading.Barrier(n, timeout=120)
        self.bufs = {}
        self.calls = 0

    def fn(self, rank):
        import torch
        from stkfmm_b200.stkfmm import device_view

        def allreduce(ptr, n, stream):
            torch.cuda.ExternalStream(int(stream)).synchronize()
            mine = device_view(ptr, n).cpu().numpy()
            self.bufs[rank] = mine
            self.bar.wait()
            total = sum(self.bufs[r] for r in range(self.n))
            self.bar.wait()
            device_view(ptr, n).copy_(torch.as_tensor(total))
            torch.cuda.synchronize()
            self.calls += 1
            return 0
        return allreduce


def run_split(pts, slv, dlv, kernel, pbc, p, max_pts, nranks, prec=0):
    """Every rank a host thread with its own handle (set_shard + set_allreduce)."""
    import threading
    import stkfmm_b200 as S
    g = HostGroup(nranks)
    outs, errs = [None] * nranks, []

    def rank(r):
        try:
            f = S.Stk3DFMM(p, max_pts, pbc, kernel, precision=prec)
            f.set_box(np.zeros(3), 1.0)
            f.set_points(pts, pts, pts if dlv is not None else None)
            f.set_shard(r, nranks)
            f.set_allreduce(g.fn(r))
            f.setup_tree(kernel)
            o = np.zeros((len(pts), S.get_kernel_dimension(kernel)[2]))
            f.evaluate_fmm(kernel, slv, o, dlv)
            outs[r] = o
        except Exception as e:  # pragma: no cover - reported below
            errs.append(e)
    ts = [threading.Thread(target=rank, args=(r,)) for r in range(nranks)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=300)
    assert not errs, errs
    return outs, g.calls


@pytest.mark.parametrize("nranks", [2, 3])
@pytest.mark.parametrize("pbc", [0, 3])
def test_far_field_split_sums_to_whole(torch_cuda, nranks, pbc):
    """With a collective, every rank runs only its share of the M2L / S2L too; the
    ranks' outputs still sum to the unsharded FMM (FP64; the downward densities are
    summed in a different order, so to rounding, not bitwise)."""
    import stkfmm_b200 as S
    rng = np.random.default_rng(40 + pbc)
    n = 6000
    pts = rng.random((n, 3)) if pbc else np.minimum(clustered_points(rng, n, nclusters=5, sigma=0.05), 0.999)
    q = rng.uniform(-0.5, 0.5, (n, 1))
    q -= q.mean()
    d = rng.normal(size=(n, 3))
    f = S.Stk3DFMM(8, 50, pbc, 1)
    f.set_box(np.zeros(3), 1.0)
    f.set_points(pts, pts, pts)
    f.setup_tree(1)
    whole = np.zeros((n, 4))
    f.evaluate_fmm(1, q, whole, d)
    parts, calls = run_split(pts, q, d, 1, pbc, 8, 50, nranks)
    assert calls == nranks  # one collective per rank and evaluation
    assert rel_l2(sum(parts), whole) < 1e-12
    # every rank did only part of the work: no rank's output alone is the whole
    assert all(rel_l2(p_, whole) > 1e-3 for p_ in parts)
