"""GPU: the hand-written adjoint of the regularized-Stokeslet P2P (StokesRegVel).

Checked against the oracle's adjoint, against FP64 torch autograd of a plain
torch restatement of the same sum, and against central finite differences
(h = 1e-6, FP64) on a subset of the points; the bar for the finite-difference
agreement is 1e-5.
"""
import math

import numpy as np
import pytest

from conftest import rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need a CUDA device"
    return t


def make_case(n, seed, eps=1e-3, sep_trg=0):
    rng = np.random.default_rng(seed)
    src = rng.random((n, 3))
    fe = np.concatenate([rng.normal(size=(n, 3)), np.full((n, 1), eps)], axis=1)
    trg = src if sep_trg == 0 else np.concatenate([src[: n // 4], rng.random((sep_trg, 3))])
    w = rng.normal(size=(len(trg), 3))
    return src, fe, trg, w


def torch_regvel(torch, src, fe, trg, pairs=None):
    """Plain torch restatement of the stokes_regvel sum (all pairs, or listed pairs)."""
    if pairs is None:
        r = trg[:, None, :] - src[None, :, :]
        f = fe[None, :, :3]
        e2 = fe[None, :, 3] ** 2
        r2 = (r * r).sum(-1)
        R2 = r2 + e2
        Rinv3 = torch.where(R2 > 0, R2.clamp_min(1e-300) ** -1.5, torch.zeros_like(R2))
        fdr = (f * r).sum(-1)
        u = ((r2 + 2 * e2)[..., None] * f + r * fdr[..., None]) * Rinv3[..., None]
        return u.sum(1) / (8 * math.pi)
    ti, si, sh = pairs
    r = trg[ti] - (src[si] + sh)
    f = fe[si, :3]
    e2 = fe[si, 3] ** 2
    r2 = (r * r).sum(-1)
    R2 = r2 + e2
    Rinv3 = R2 ** -1.5
    fdr = (f * r).sum(-1)
    u = ((r2 + 2 * e2)[:, None] * f + r * fdr[:, None]) * Rinv3[:, None] / (8 * math.pi)
    out = torch.zeros((len(trg), 3), dtype=u.dtype, device=u.device)
    return out.index_add(0, ti, u)


def dev(torch, a, grad=False):
    return torch.tensor(np.asarray(a), dtype=torch.float64, device="cuda", requires_grad=grad)


@pytest.mark.parametrize("prec,tol", [(0, 1e-12), (1, 1e-6)])
def test_adjoint_direct_matches_oracle(torch, prec, tol):
    from stkfmm_b200.autograd import stokes_regvel
    src, fe, trg, w = make_case(1500, 1, eps=2e-3, sep_trg=900)
    gf_ref, gx_ref = O.regvel_adjoint(src, fe, trg, w)
    xs, v, xt = dev(torch, src, True), dev(torch, fe, True), dev(torch, trg, True)
    u = stokes_regvel(xs, v, xt, precision=prec)
    u.backward(dev(torch, w))
    assert rel_l2(v.grad[:, :3].cpu().numpy(), gf_ref) < tol
    assert rel_l2(xs.grad.cpu().numpy(), gx_ref) < tol
    ref = O.direct(O.UK_STOKES_REGVEL, src, fe, trg)
    assert rel_l2(u.detach().cpu().numpy(), ref) < tol


def test_adjoint_direct_matches_torch_autograd(torch):
    """Every gradient (f, eps, source and target positions) against FP64 torch autograd."""
    from stkfmm_b200.autograd import stokes_regvel
    src, fe, trg, w = make_case(800, 2, eps=5e-3, sep_trg=700)
    fe[:, 3] = np.random.default_rng(3).uniform(1e-3, 1e-2, len(fe))
    a = [dev(torch, x, True) for x in (src, fe, trg)]
    b = [dev(torch, x, True) for x in (src, fe, trg)]
    wt = dev(torch, w)
    stokes_regvel(*a).backward(wt)
    (torch_regvel(torch, *b) * wt).sum().backward()
    for ga, gb in zip(a, b):
        assert rel_l2(ga.grad.cpu().numpy(), gb.grad.cpu().numpy()) < 1e-12


def test_adjoint_finite_differences(torch):
    """Central differences, h = 1e-6, FP64, at 8 points of a subset: per point, the relative
    error |fd - g| / |fd| of the 3-vector gradient (no absolute floor)."""
    from stkfmm_b200.autograd import stokes_regvel
    src, fe, _, w = make_case(4096, 4, eps=1e-3)
    xs, v = dev(torch, src, True), dev(torch, fe, True)
    wt = dev(torch, w)
    u = stokes_regvel(xs, v, xs)
    (u * wt).sum().backward()
    gx, gv = xs.grad.cpu().numpy(), v.grad.cpu().numpy()

    def loss(s, val):
        with torch.no_grad():
            return float((stokes_regvel(dev(torch, s), dev(torch, val), dev(torch, s)) * wt).sum())

    h = 1e-6
    rng = np.random.default_rng(5)
    worst = 0.0
    for i in rng.choice(len(src), 8, replace=False):
        fdx, fdv = np.zeros(3), np.zeros(3)
        for k in range(3):
            sp, sm = src.copy(), src.copy()
            sp[i, k] += h
            sm[i, k] -= h
            fdx[k] = (loss(sp, fe) - loss(sm, fe)) / (2 * h)
            vp, vm = fe.copy(), fe.copy()
            vp[i, k] += h
            vm[i, k] -= h
            fdv[k] = (loss(src, vp) - loss(src, vm)) / (2 * h)
        worst = max(worst, np.linalg.norm(fdx - gx[i]) / np.linalg.norm(fdx),
                    np.linalg.norm(fdv - gv[i, :3]) / np.linalg.norm(fdv))
    assert worst < 1e-5, worst


@pytest.mark.parametrize("pbc", [0, 3])
def test_adjoint_ulist_matches_torch_autograd(torch, pbc):
    """Near-field (U-list) pairs, periodic or not, against torch autograd of the listed pairs."""
    from stkfmm_b200 import Octree
    from stkfmm_b200.autograd import UListPlan, stokes_regvel
    rng = np.random.default_rng(6 + pbc)
    n = 2500
    pts = rng.random((n, 3))
    fe = np.concatenate([rng.normal(size=(n, 3)), rng.uniform(1e-3, 4e-3, (n, 1))], axis=1)
    w = rng.normal(size=(n, 3))
    plan = UListPlan(pts, max_pts=40, pbc=pbc)
    # explicit pair list from the same U-list
    t = Octree(pts, 40, pbc, sl=pts, trg=pts)
    perm, b, e = t.point_set(0)
    off, ent = t.list("U")
    ti, si, sh = [], [], []
    for box in range(t.num_nodes):
        tgt = perm[b[box]:e[box]]
        for en in ent[off[box]:off[box + 1]]:
            sb, code = en >> 5, en & 31
            src_pts = perm[b[sb]:e[sb]]
            shift = np.array([code % 3 - 1, (code // 3) % 3 - 1, code // 9 - 1], dtype=np.float64)
            tt, ss = np.meshgrid(tgt, src_pts, indexing="ij")
            ti.append(tt.ravel())
            si.append(ss.ravel())
            sh.append(np.repeat(shift[None], tt.size, axis=0))
    pairs = (torch.as_tensor(np.concatenate(ti)).cuda(), torch.as_tensor(np.concatenate(si)).cuda(),
             torch.as_tensor(np.concatenate(sh)).cuda())
    a = [dev(torch, x, True) for x in (pts, fe)]
    b_ = [dev(torch, x, True) for x in (pts, fe)]
    wt = dev(torch, w)
    u = stokes_regvel(a[0], a[1], a[0], plan=plan)
    ref_u = torch_regvel(torch, b_[0], b_[1], b_[0], pairs=pairs)
    assert rel_l2(u.detach().cpu().numpy(), ref_u.detach().cpu().numpy()) < 1e-12
    (u * wt).sum().backward()
    (ref_u * wt).sum().backward()
    for ga, gb in zip(a, b_):
        assert rel_l2(ga.grad.cpu().numpy(), gb.grad.cpu().numpy()) < 1e-12


def test_adjoint_mixed_close_to_fp64(torch):
    from stkfmm_b200.autograd import UListPlan, stokes_regvel
    rng = np.random.default_rng(8)
    n = 20000
    pts = rng.random((n, 3))
    fe = np.concatenate([rng.normal(size=(n, 3)), np.full((n, 1), 1e-3)], axis=1)
    w = dev(torch, rng.normal(size=(n, 3)))
    plan = UListPlan(pts, max_pts=64)
    grads = []
    for prec in (0, 1):
        x, v = dev(torch, pts, True), dev(torch, fe, True)
        (stokes_regvel(x, v, x, plan=plan, precision=prec) * w).sum().backward()
        grads.append((x.grad.cpu().numpy(), v.grad.cpu().numpy()))
    assert rel_l2(grads[1][0], grads[0][0]) < 1e-6
    assert rel_l2(grads[1][1], grads[0][1]) < 1e-6
