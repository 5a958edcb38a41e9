"""Host-side argument checks of the differentiable RegVel P2P (no GPU needed: the
checks run before any device work; the U-list plan's tree is the host-only octree)."""
import numpy as np
import pytest
import torch

from stkfmm_b200.autograd import UListPlan, stokes_regvel


def _case(n=400, seed=0):
    rng = np.random.default_rng(seed)
    pts = rng.random((n, 3))
    fe = np.concatenate([rng.normal(size=(n, 3)), np.full((n, 1), 1e-3)], axis=1)
    return pts, torch.as_tensor(pts), torch.as_tensor(fe)


def test_ulist_plan_rejects_other_targets():
    pts, x, v = _case()
    plan = UListPlan(pts, max_pts=32)
    other = x + 0.25
    with pytest.raises(ValueError, match="trg_xyz must be the source points"):
        stokes_regvel(x, v, other, plan=plan)


def test_ulist_plan_rejects_other_point_count():
    pts, x, v = _case()
    plan = UListPlan(pts, max_pts=32)
    with pytest.raises(ValueError, match="UListPlan of 400 points"):
        stokes_regvel(x[:300], v[:300], x[:300], plan=plan)
