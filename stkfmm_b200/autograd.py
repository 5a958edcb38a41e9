"""Differentiable regularized-Stokeslet P2P (StokesRegVel) behind torch.autograd.

Forward, as the reference's stokes_regvel kernel
(Lib/include/STKFMM/StokesRegSingleLayerKernel.hpp:17-41):

    u_t = 1/(8 pi) sum_s G_{eps_s}(x_t - x_s) f_s,
    G_eps(r) = ((|r|^2 + 2 eps^2) I + r r^T) / (|r|^2 + eps^2)^{3/2}

over all (target, source) pairs ("direct") or over the U-list pairs of an
adaptive octree ("ulist", sources = targets).  The backward pass is a
hand-written adjoint P2P kernel pair run through the C ABI; it recomputes the
pair terms instead of storing them:

    STK_UK_REGVEL_ADJ_SRC: dL/df_s, dL/deps_s, dL/dx_s  (outputs at the sources,
                           inputs = the targets with w_t = dL/du_t)
    STK_UK_REGVEL_ADJ_TRG: dL/dx_t                      (outputs at the targets)

No reference counterpart: STKFMM has no differentiation.  torch only holds the
device memory and the stream; every pair sum runs in libstkfmm_b200.so.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import P_i, check, lib
from .stkfmm import Octree, PRECISION, UKERNEL


def _stream():
    return torch.cuda.current_stream().cuda_stream


def _c(t):
    return t.detach().to(dtype=torch.float64).contiguous()


class DirectPlan:
    """All (target, source) pairs: FMMData::evaluateKernel semantics."""

    mode = "direct"

    def forward(self, src, sval, trg, out, prec):
        check(lib().stk_ukernel_direct_device(int(UKERNEL.STOKES_REGVEL), len(src), src.data_ptr(), sval.data_ptr(),
                                              len(trg), trg.data_ptr(), out.data_ptr(), int(prec), _stream()),
              "regvel forward")

    def adjoint_src(self, src, sval, trg, w, gsrc, prec):
        # outputs at the sources (values f, eps), inputs at the targets (values w)
        check(lib().stk_ukernel_direct_aux_device(int(UKERNEL.REGVEL_ADJ_SRC), len(trg), trg.data_ptr(), w.data_ptr(),
                                                  len(src), src.data_ptr(), sval.data_ptr(), gsrc.data_ptr(),
                                                  int(prec), _stream()), "regvel adjoint (sources)")

    def adjoint_trg(self, src, sval, trg, w, gtrg, prec):
        check(lib().stk_ukernel_direct_aux_device(int(UKERNEL.REGVEL_ADJ_TRG), len(src), src.data_ptr(),
                                                  sval.data_ptr(), len(trg), trg.data_ptr(), w.data_ptr(),
                                                  gtrg.data_ptr(), int(prec), _stream()), "regvel adjoint (targets)")


class UListPlan:
    """Near-field pairs only: the U-list of an adaptive octree over one point set
    (sources = targets), max_pts points per leaf, coordinates in [0,1)^3.  The list
    is uploaded once into a device plan (stk_p2p_plan_create) that the forward and
    both adjoint passes execute asynchronously on torch's current stream."""

    mode = "ulist"

    def __init__(self, points, max_pts=64, pbc=0):
        pts = np.ascontiguousarray(np.asarray(points, dtype=np.float64).reshape(-1, 3))
        self.tree = Octree(pts, max_pts, pbc, sl=pts, trg=pts)
        perm, beg, end = self.tree.point_set(0)
        tperm, tb, te = self.tree.point_set(2)
        assert np.array_equal(perm, tperm)
        off, ent = self.tree.list("U")
        self.n = len(pts)
        # The adjoint of "target box A sees source box B through image shift s" is
        # "output box B sees input box A through shift -s"; U(B) holds exactly (A, -s),
        # so the U-list serves as its own transpose.
        self.arrs = [np.ascontiguousarray(a, dtype=np.int32) for a in (tb, te, off, ent, beg, end)]
        self.perm = None
        self._perm_np = perm
        self._plan = None
        self._plan_dev = None

    def __del__(self):
        if getattr(self, "_plan", None):
            lib().stk_p2p_plan_destroy(self._plan)
            self._plan = None

    def plan(self, device):
        """The device plan of the U list (created on first use, on `device`)."""
        if self._plan is None or self._plan_dev != device:
            if self._plan:
                lib().stk_p2p_plan_destroy(self._plan)
            tb, te, off, ent, beg, end = self.arrs
            st = np.zeros(1, np.int32)
            with torch.cuda.device(device):
                self._plan = lib().stk_p2p_plan_create(len(tb), *(a.ctypes.data_as(P_i) for a in (tb, te, off, ent)),
                                                       len(beg), beg.ctypes.data_as(P_i), end.ctypes.data_as(P_i),
                                                       self.n, self.n, 1.0, st.ctypes.data_as(P_i))
            if not self._plan:
                check(int(st[0]) or 5, "stk_p2p_plan_create")
            self._plan_dev = device
        return self._plan

    def pairs(self):
        """(target, source point) pairs of one pass over the U list."""
        return int(lib().stk_p2p_plan_pairs(self.plan(torch.device("cuda", torch.cuda.current_device()))))

    def _p(self, device):
        if self.perm is None or self.perm.device != device:
            self.perm = torch.as_tensor(self._perm_np.astype(np.int64), device=device)
        return self.perm

    def _run(self, uk, src_s, val_s, trg_s, aux_s, out_s, prec):
        pl = self.plan(src_s.device)
        rc = lib().stk_p2p_plan_execute(pl, int(uk), int(prec), src_s.data_ptr(), val_s.data_ptr(), trg_s.data_ptr(),
                                        aux_s.data_ptr() if aux_s is not None else None, out_s.data_ptr(), _stream())
        check(rc, "regvel ulist")

    def _sorted(self, *ts):
        p = self._p(ts[0].device)
        return [t[p].contiguous() for t in ts]

    def _unsort(self, t_sorted, out):
        out[self._p(t_sorted.device)] = t_sorted

    def forward(self, src, sval, trg, out, prec):
        src_s, val_s = self._sorted(src, sval)
        o = torch.zeros_like(out)
        self._run(UKERNEL.STOKES_REGVEL, src_s, val_s, src_s, None, o, prec)
        self._unsort(o, out)

    def adjoint_src(self, src, sval, trg, w, gsrc, prec):
        src_s, val_s, w_s = self._sorted(src, sval, w)
        o = torch.zeros_like(gsrc)
        self._run(UKERNEL.REGVEL_ADJ_SRC, src_s, w_s, src_s, val_s, o, prec)
        self._unsort(o, gsrc)

    def adjoint_trg(self, src, sval, trg, w, gtrg, prec):
        src_s, val_s, w_s = self._sorted(src, sval, w)
        o = torch.zeros_like(gtrg)
        self._run(UKERNEL.REGVEL_ADJ_TRG, src_s, val_s, src_s, w_s, o, prec)
        self._unsort(o, gtrg)


class StokesRegVelP2P(torch.autograd.Function):
    """u = RegVel P2P(src_xyz, src_val = (f, eps), trg_xyz) with a hand-written adjoint."""

    @staticmethod
    def forward(ctx, src_xyz, src_val, trg_xyz, plan, precision):
        src, sval, trg = _c(src_xyz), _c(src_val), _c(trg_xyz)
        if plan.mode == "ulist":
            # the U list is of one point set: its targets are its sources
            if len(src) != plan.n or len(sval) != plan.n:
                raise ValueError("UListPlan of %d points given %d sources" % (plan.n, len(src)))
            if trg.data_ptr() != src.data_ptr() and not (trg.shape == src.shape and torch.equal(trg, src)):
                raise ValueError("UListPlan: trg_xyz must be the source points")
        out = torch.zeros((len(trg), 3), dtype=torch.float64, device=src.device)
        plan.forward(src, sval, trg, out, precision)
        ctx.save_for_backward(src, sval, trg)
        ctx.plan, ctx.precision = plan, precision
        return out

    @staticmethod
    def backward(ctx, grad_u):
        src, sval, trg = ctx.saved_tensors
        w = _c(grad_u)
        gsrc = torch.zeros((len(src), 7), dtype=torch.float64, device=src.device)
        ctx.plan.adjoint_src(src, sval, trg, w, gsrc, ctx.precision)
        gtrg = torch.zeros((len(trg), 3), dtype=torch.float64, device=src.device)
        ctx.plan.adjoint_trg(src, sval, trg, w, gtrg, ctx.precision)
        return gsrc[:, 4:7], gsrc[:, 0:4], gtrg, None, None


def stokes_regvel(src_xyz, src_val, trg_xyz=None, plan=None, precision=PRECISION.FP64):
    """Differentiable regularized-Stokeslet velocity at the targets (CUDA tensors).

    src_val holds (f_x, f_y, f_z, eps) per source.  Without a plan the sum runs
    over all pairs; UListPlan(points) restricts it to the octree's near field
    (then trg_xyz must be the same points as src_xyz).  Gradients flow to
    src_xyz, src_val (f and eps) and trg_xyz.
    """
    if trg_xyz is None:
        trg_xyz = src_xyz
    if plan is None:
        plan = DirectPlan()
    return StokesRegVelP2P.apply(src_xyz, src_val, trg_xyz, plan, int(precision))
