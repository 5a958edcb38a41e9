"""GPU parity at the benchmark workloads' full sizes, through the library's public API.

The smaller parity tests compare whole outputs with the oracle on trees of a
few thousand points.  Here the workloads the benchmark times run at their full
sizes, and what the oracle can afford is checked exactly; the rest is covered by
size-independent properties:

* LapPGrad U-list S2T (SL + DL at the same points), 1,048,576 points in 64
  Gaussian clusters (sigma 0.02), max 256 points per leaf: the FP64 output
  against the oracle over randomly sampled target leaves (their full U lists),
  1e-12 relative L2; the mixed output against the FP64 output over all targets,
  1e-6; repeated evaluations bitwise identical in both precisions.
* StokesVel free-space FMM, 32,768 uniform points, p = 8, max 128 points per
  leaf: FP64 and mixed against the oracle's direct sum at 4,096 sampled
  targets, with the per-component bar the FMM tests use at p = 8.
* Differentiated StokesRegVel U-list P2P, 1,048,576 uniform points, eps = 1e-3:
  d loss/d x and d loss/d f against central differences (h = 1e-6, FP64) of
  the full loss at sampled points, per point, without an absolute floor; mixed
  gradients against FP64 ones.
"""
import numpy as np
import pytest

from conftest import component_errors, rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu

LAPPGRAD, STOKES = 1, 8  # KERNEL enum values (STKFMM_common.hpp)


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    torch.cuda.set_device(0)
    return torch


def clustered_1m(seed=0):
    """1,048,576 points from 64 Gaussian clusters (centres U[0.1,0.9]^3, sigma 0.02),
    clipped to [0,1)^3; q ~ U(-0.5,0.5), d ~ N(0,1)^3."""
    rng = np.random.default_rng(seed)
    n = 1 << 20
    centres = rng.uniform(0.1, 0.9, size=(64, 3))
    idx = rng.integers(0, 64, size=n)
    pts = np.clip(centres[idx] + rng.normal(0.0, 0.02, size=(n, 3)), 0.0, np.nextafter(1.0, 0.0))
    return pts, rng.uniform(-0.5, 0.5, size=(n, 1)), rng.normal(size=(n, 3))


def sampled_leaves(ul, budget_pairs, seed):
    """Random target leaves with non-empty U lists whose pairs add up to ~budget_pairs."""
    tb, te, off, ent = ul["trg_begin"], ul["trg_end"], ul["list_off"], ul["list_ent"]
    cnt = ul["sl_end"] - ul["sl_begin"]
    nt = te - tb
    ns = np.array([cnt[ent[off[b]:off[b + 1]] >> 5].sum() for b in range(len(tb))], dtype=np.int64)
    cand = np.flatnonzero((nt > 0) & (ns > 0))
    rng = np.random.default_rng(seed)
    rng.shuffle(cand)
    pick, tot = [], 0
    for b in cand:
        pick.append(b)
        tot += int(nt[b]) * int(ns[b])
        if tot >= budget_pairs:
            break
    return np.array(sorted(pick), dtype=np.int64)


def test_lappgrad_clustered_1m_ulist(torch_cuda):
    import stkfmm_b200 as S
    torch = torch_cuda
    pts, q, d = clustered_1m()
    n = len(pts)
    fmm = S.Stk3DFMM(10, 256, S.PAXIS.NONE, LAPPGRAD)
    fmm.set_box(np.zeros(3), 1.0)
    fmm.set_points(pts, pts, pts)
    fmm.setup_tree(LAPPGRAD)
    qd, dd = torch.as_tensor(q).cuda(), torch.as_tensor(d).cuda()
    outs = {}
    for prec in (S.PRECISION.FP64, S.PRECISION.MIXED):
        fmm.set_precision(prec)
        runs = []
        for _ in range(2):
            out = torch.zeros((n, 4), dtype=torch.float64, device="cuda")
            fmm.evaluate_near_device(LAPPGRAD, qd.data_ptr(), out.data_ptr(), dd.data_ptr())
            torch.cuda.synchronize()
            runs.append(out.cpu().numpy())
        assert np.array_equal(runs[0], runs[1]), ("repeat differs", prec)
        outs[int(prec)] = runs[0]
    o64, omx = outs[int(S.PRECISION.FP64)], outs[int(S.PRECISION.MIXED)]
    assert np.isfinite(o64).all() and np.isfinite(omx).all()
    assert rel_l2(omx, o64) < 1e-6, rel_l2(omx, o64)

    # the oracle over the full U lists of sampled target leaves
    ul = fmm.ulist(LAPPGRAD)
    boxes = sampled_leaves(ul, 1.5e7, seed=3)
    tb, te = ul["trg_begin"][boxes], ul["trg_end"][boxes]
    off = np.concatenate([[0], np.cumsum(ul["list_off"][boxes + 1] - ul["list_off"][boxes])])
    ent = np.concatenate([ul["list_ent"][ul["list_off"][b]:ul["list_off"][b + 1]] for b in boxes])
    sp, tp, dp = ul["sl_perm"], ul["trg_perm"], ul["dl_perm"]
    trg = pts[tp]
    ref = (O.lists(O.UK_LAPLACE_PGRAD, tb, te, off, ent >> 5, ent & 31, ul["sl_begin"], ul["sl_end"], pts[sp], q[sp],
                   trg)
           + O.lists(O.UK_LAPLACE_DIPOLEPGRAD, tb, te, off, ent >> 5, ent & 31, ul["dl_begin"], ul["dl_end"], pts[dp],
                     d[dp], trg))
    sel = np.concatenate([np.arange(a, b) for a, b in zip(tb, te)])
    assert len(sel) > 1000
    err = rel_l2(o64[tp[sel]], ref[sel])
    assert err < 1e-12, err
    assert rel_l2(omx[tp[sel]], ref[sel]) < 1e-6


def test_stokes_32k_fmm_vs_direct_sum(torch_cuda):
    import stkfmm_b200 as S
    rng = np.random.default_rng(0)
    n = 32768
    pts = rng.random((n, 3))
    f = rng.normal(size=(n, 3))
    samp = np.sort(np.random.default_rng(11).choice(n, 4096, replace=False))
    ref = O.direct(O.UK_STOKES_VEL, pts, f, pts[samp])
    fmm = S.Stk3DFMM(8, 128, S.PAXIS.NONE, STOKES)
    fmm.set_box(np.zeros(3), 1.0)
    fmm.set_points(pts, pts, None)
    fmm.setup_tree(STOKES)
    for prec in (S.PRECISION.FP64, S.PRECISION.MIXED):
        fmm.set_precision(prec)
        out = np.zeros((n, 3))
        fmm.evaluate_fmm(STOKES, f, out, None)
        errs = component_errors(out[samp], ref)
        assert max(errs) < 2e-5, (prec, errs)


def test_regvel_adjoint_1m_finite_differences(torch_cuda):
    from stkfmm_b200.autograd import UListPlan, stokes_regvel
    torch = torch_cuda
    rng = np.random.default_rng(0)
    n = 1 << 20
    pts = rng.random((n, 3))
    fe = np.concatenate([rng.normal(size=(n, 3)), np.full((n, 1), 1e-3)], axis=1)
    w = rng.normal(size=(n, 3))
    plan = UListPlan(pts, max_pts=256)
    x, v, wt = (torch.as_tensor(a).cuda() for a in (pts, fe, w))
    grads = {}
    for prec in (0, 1):
        xx = x.detach().requires_grad_(True)
        vv = v.detach().requires_grad_(True)
        (stokes_regvel(xx, vv, xx, plan=plan, precision=prec) * wt).sum().backward()
        grads[prec] = (xx.grad.cpu().numpy(), vv.grad.cpu().numpy())
    gx, gv = grads[0]
    assert rel_l2(grads[1][0], gx) < 1e-6
    assert rel_l2(grads[1][1][:, :3], gv[:, :3]) < 1e-6

    # central differences of the full loss at sampled points, over the pairs each point enters
    samp = np.sort(np.random.default_rng(21).choice(n, 1024, replace=False))
    perm, beg, end = plan.tree.point_set(0)
    off, ent = plan.tree.list("U")
    leaf_of = np.empty(n, np.int64)
    for b in np.flatnonzero(plan.tree.first_child < 0):
        leaf_of[perm[beg[b]:end[b]]] = b
    nb_off, nb = [0], []
    for i in samp:
        b = leaf_of[i]
        lst = np.concatenate([perm[beg[sb]:end[sb]] for sb in (ent[off[b]:off[b + 1]] >> 5)])
        nb.append(lst)
        nb_off.append(nb_off[-1] + len(lst))
    fdx, fdf = O.regvel_fd_local(samp, np.array(nb_off), np.concatenate(nb), pts, fe, w, h=1e-6)
    per_point_x = np.linalg.norm(gx[samp] - fdx, axis=1) / np.linalg.norm(fdx, axis=1)
    per_point_f = np.linalg.norm(gv[samp, :3] - fdf, axis=1) / np.linalg.norm(fdf, axis=1)
    assert per_point_x.max() < 1e-5, per_point_x.max()
    assert per_point_f.max() < 1e-5, per_point_f.max()
