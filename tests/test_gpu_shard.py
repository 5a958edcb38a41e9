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
