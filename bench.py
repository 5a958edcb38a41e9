#!/usr/bin/env python
"""Benchmark: STKFMM near-field P2P on B200.

Workload (one "step"): one U-list S2T pass of the LapPGrad kernel (single layer
q ~ U(-0.5,0.5) and double layer d ~ N(0,1)^3 at the same points as the
targets) over an adaptive octree of 1,048,576 points drawn from 64 Gaussian
clusters (centres U[0.1,0.9]^3, sigma 0.02, clipped into [0,1)^3), max 256
points per leaf, multipole order 10.  Seeded synthetic data stands in for the
reference's TOML-configured point sets.

Metric: P2P pair-interactions/s (SL and DL (target, source point) pairs counted
separately, exact counts from the U-list) of the plain FP64 path, the
reference's precision, as the headline; the mixed-precision path (FP64
centre-relative displacement, FP32 kernel, Kahan FP32 accumulation) beside it
with its ratio to FP64 and its error against FP64.

The reference arm (--impl reference) runs the reference's own micro-kernel
bodies (LaplaceLayerKernel.hpp laplace_pgrad + laplace_dipolepgrad, compiled in
place) in a PVFMM-style SIMD pair loop on all host cores, over the same U-list
of the same tree (built by the host-only libstk_octree.so; the GPU library is
not loaded), one full step per step.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun (N > 1) each rank runs an independent replica (its own seed) on
its own GPU: weak scaling, no collective on the data path; timing is the max
over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_POINTS = 1_048_576
N_CLUSTERS = 64
SIGMA = 0.02
MAX_PTS = 256
MULT_ORDER = 10
KERNEL_LAPPGRAD = 1
# Algorithmic flops per (target, source point) pair of the fused laplace_pgrad +
# laplace_dipolepgrad micro-kernel (FMA = 2), counted from stk_ukernels.cuh
# (Uk<UK_LAPLACE_SLDL_PGRAD>::eval): displacement 3, r^2 5, 1/r^2 1, r.d 5, w 2,
# potential 2, radial coefficient 2, 1/r^3 1, gradient 12 = 33, plus one
# reciprocal square root.  The same count serves both paths: the mixed path's
# hi/lo displacement split (9) and Newton step on the MUFU rsqrt (5), and the
# FP64 path's rsqrt refinement, are implementation work and are not counted.
FLOPS_PER_POINT_PAIR = 33
WORKLOAD = ("LapPGrad U-list P2P (S2T SL+DL), 1,048,576 pts in 64 Gaussian clusters (sigma 0.02, centres "
            "U[0.1,0.9]^3), max 256 pts/leaf, p=10, SL=DL=targets")
WORKLOAD_FMM = ("LapPGrad free-space FMM (evaluate_fmm: U/W/X near field + KIFMM far field), same points and "
                "values, p=10, max 256 pts/leaf")
FMM_SAMPLE = 4096  # targets of the FMM accuracy check against the direct sum
METRIC = "P2P pair-interactions/s (U-list S2T SL+DL; FP64 path, mixed beside it; FMM evals/s in fmm)"


def make_points(seed: int):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.1, 0.9, size=(N_CLUSTERS, 3))
    idx = rng.integers(0, N_CLUSTERS, size=N_POINTS)
    pts = centres[idx] + rng.normal(0.0, SIGMA, size=(N_POINTS, 3))
    pts = np.clip(pts, 0.0, np.nextafter(1.0, 0.0))
    q = rng.uniform(-0.5, 0.5, size=(N_POINTS, 1))
    d = rng.normal(size=(N_POINTS, 3))
    return pts, q, d


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(vals, ws, device="cuda"):
    """Element-wise max of per-rank timings over the process group (identity for one rank)."""
    if ws <= 1:
        return [float(v) for v in vals]
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def job_rate(units_per_rank, ws, seconds):
    """Whole-job throughput: every rank processes units_per_rank in (max over ranks) seconds."""
    return ws * units_per_rank / seconds


# ---------------------------------------------------------------- clocks ----
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------- further FMM workloads ----
EXTRA_FMM = [
    {"name": "stokes_32k_uniform", "kernel": 8, "pbc": 0, "p": 8, "max_pts": 128, "n": 32768,
     "workload": "StokesVel free-space FMM: 32,768 points ~ U[0,1)^3 as sources and targets, f ~ N(0,1)^3, "
                 "p=8, max 128 pts/leaf, seed 0"},
    {"name": "rpy_pxyz_2m_uniform", "kernel": 16, "pbc": 3, "p": 8, "max_pts": 256, "n": 2097152,
     "workload": "RPY triply periodic (PXYZ) FMM: 2,097,152 points ~ U[0,1)^3, f ~ N(0,1)^3 minus its mean, "
                 "b ~ U(1e-4,5e-4), p=8, max 256 pts/leaf, seed 0"},
    {"name": "pvel_pxy_4m_spheres", "kernel": 128, "pbc": 2, "p": 12, "max_pts": 512, "n": 4194304,
     "workload": "StokesPVel doubly periodic (PXY) FMM, single and double layer: 4,194,304 points on the surfaces "
                 "of 4,096 spheres (radius 0.01, centres ~ U([0.05,0.95]^2 x [0.05,0.5])), f ~ N(0,1)^3 with "
                 "trD = 0 and the mean of (f, trD) removed, D ~ N(0,1)^9 with its mean trace removed, p=12, "
                 "max 512 pts/leaf, seed 0"},
]


# no-slip wall (StkWallFMM): sources = targets, 64 Gaussian clusters in x, y, heights in [0.01, 0.49]
WALL_FMM = [
    {"name": "wall_stokes_1m_clustered", "kernel": 8, "pbc": 0, "p": 8, "max_pts": 256, "n": 1048576,
     "workload": "StkWallFMM Stokeslets above a no-slip wall (free space): 1,048,576 points in 64 Gaussian "
                 "clusters (sigma 0.02, centres U[0.1,0.9]^3) with heights mapped to [0.01, 0.49] of the unit box "
                 "(wall at z = 0), sources = targets, f ~ N(0,1)^3, p=8, max 256 pts/leaf, seed 0"},
    {"name": "wall_rpy_1m_clustered", "kernel": 16, "pbc": 0, "p": 8, "max_pts": 256, "n": 1048576,
     "workload": "StkWallFMM RPY spheres above a no-slip wall (free space): the same 1,048,576 points, f ~ N(0,1)^3, "
                 "b ~ U(1e-4, 5e-4), p=8, max 256 pts/leaf, seed 0"},
]


# differentiated StokesRegVel (hand-written adjoint P2P behind torch.autograd)
ADJ = {"name": "regvel_adjoint_1m_uniform", "n": 1_048_576, "eps": 1e-3, "max_pts": 256, "fd_sample": 4096,
       "fd_h": 1e-6,
       "workload": "Differentiated StokesRegVel U-list P2P: 1,048,576 points ~ U[0,1)^3 as sources and targets, "
                   "f ~ N(0,1)^3, eps = 1e-3 per source, loss = sum_t w_t . u_t with w ~ N(0,1)^3, max 256 pts/leaf, "
                   "seed 0; one step = forward + hand-written adjoint (d loss/d f, d loss/d eps, d loss/d x)"}


def regvel_torch(torch, src, fe, trg):
    """Plain torch restatement of the stokes_regvel direct sum (all pairs), for FP64 autograd."""
    import math
    r = trg[:, None, :] - src[None, :, :]
    f = fe[None, :, :3]
    e2 = fe[None, :, 3] ** 2
    r2 = (r * r).sum(-1)
    R2 = r2 + e2
    Rinv3 = R2 ** -1.5
    fdr = (f * r).sum(-1)
    u = ((r2 + 2 * e2)[..., None] * f + r * fdr[..., None]) * Rinv3[..., None]
    return u.sum(1) / (8 * math.pi)


def time_adjoint(steps, warmup, seed, ws, flush):
    """Forward + adjoint of the StokesRegVel U-list P2P through torch.autograd, FP64 and mixed,
    CUDA events per step (torch's stream); gradients kept for the checks."""
    import torch
    from stkfmm_b200.autograd import UListPlan, stokes_regvel
    rng = np.random.default_rng(seed)
    n = ADJ["n"]
    pts = rng.random((n, 3))
    fe = np.concatenate([rng.normal(size=(n, 3)), np.full((n, 1), ADJ["eps"])], axis=1)
    w = rng.normal(size=(n, 3))
    t0 = time.perf_counter()
    plan = UListPlan(pts, max_pts=ADJ["max_pts"])
    pairs = plan.pairs()
    res = {"workload": ADJ["workload"], "setup_tree_s": time.perf_counter() - t0, "pairs_per_pass": pairs,
           "pairs_per_step": 3 * pairs,
           "step": "forward (stokes_regvel) + adjoint sources (d/df, d/deps, d/dx_s) + adjoint targets (d/dx_t), "
                   "each one pass over the U-list pairs"}
    x = torch.as_tensor(pts).cuda()
    v = torch.as_tensor(fe).cuda()
    wt = torch.as_tensor(w).cuda()
    grads = {}
    for prec, nm in ((0, "fp64"), (1, "mixed")):
        def step():
            xx = x.detach().requires_grad_(True)
            vv = v.detach().requires_grad_(True)
            u = stokes_regvel(xx, vv, xx, plan=plan, precision=prec)
            (u * wt).sum().backward()
            return xx, vv
        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        ms = []
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            xx, vv = step()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        m = max_over_ranks([sum(ms) / len(ms)], ws)[0]
        res[nm] = {"pairs_per_s": job_rate(3 * pairs, ws, m * 1e-3), "ms_per_step": m}
        grads[nm] = (xx.grad.cpu().numpy(), vv.grad.cpu().numpy())
    res["mixed_over_fp64"] = res["fp64"]["ms_per_step"] / res["mixed"]["ms_per_step"]
    res["rel_l2_mixed_vs_fp64"] = {
        "d_dx": float(np.linalg.norm(grads["mixed"][0] - grads["fp64"][0]) / np.linalg.norm(grads["fp64"][0])),
        "d_df": float(np.linalg.norm(grads["mixed"][1][:, :3] - grads["fp64"][1][:, :3])
                      / np.linalg.norm(grads["fp64"][1][:, :3]))}
    res["timing"] = "CUDA events around forward + backward on torch's stream, L2 flushed between steps"
    res["_chk"] = (pts, fe, w, plan, grads["fp64"])
    return res


def adjoint_checks(res):
    """Central finite differences (FP64, h = 1e-6) of the 1M-point loss at a 4,096-point sample
    (oracle, over the pairs each sampled point enters), and FP64 torch autograd of the direct sum
    over a 4,096-point subset."""
    import torch
    from oracle import oracle as O
    from stkfmm_b200.autograd import stokes_regvel
    O.build()
    pts, fe, w, plan, (gx, gv) = res.pop("_chk")
    n = len(pts)
    samp = np.sort(np.random.default_rng(21).choice(n, ADJ["fd_sample"], replace=False))
    # each sampled point's partners: the points of the leaves in its leaf's U list (U is symmetric)
    perm, beg, end = plan.tree.point_set(0)
    off, ent = plan.tree.list("U")
    leaf_of = np.empty(n, np.int64)
    isleaf = plan.tree.first_child < 0
    for b in np.flatnonzero(isleaf):
        leaf_of[perm[beg[b]:end[b]]] = b
    nb_off, nb = [0], []
    for i in samp:
        b = leaf_of[i]
        lst = np.concatenate([perm[beg[sb]:end[sb]] for sb in (ent[off[b]:off[b + 1]] >> 5)])
        nb.append(lst)
        nb_off.append(nb_off[-1] + len(lst))
    t0 = time.perf_counter()
    fdx, fdf = O.regvel_fd_local(samp, np.array(nb_off), np.concatenate(nb), pts, fe, w, h=ADJ["fd_h"])
    fd_s = time.perf_counter() - t0
    gxs, gfs = gx[samp], gv[samp, :3]
    per_point = lambda g, fd: float(np.max(np.linalg.norm(g - fd, axis=1) / np.linalg.norm(fd, axis=1)))
    res["finite_differences"] = {
        "sample": "%d points drawn with seed 21 from the 1,048,576; central differences h = %g in FP64 by the oracle "
                  "over the pairs each point enters (%.1f s)" % (len(samp), ADJ["fd_h"], fd_s),
        "rel_l2_d_dx": float(np.linalg.norm(gxs - fdx) / np.linalg.norm(fdx)),
        "rel_l2_d_df": float(np.linalg.norm(gfs - fdf) / np.linalg.norm(fdf)),
        "max_per_point_rel_d_dx": per_point(gxs, fdx),
        "max_per_point_rel_d_df": per_point(gfs, fdf),
        "bar": 1e-5}
    # FP64 torch autograd of the direct sum over a 4,096-point subset
    sub = samp
    a = [torch.tensor(z, dtype=torch.float64, device="cuda", requires_grad=True) for z in (pts[sub], fe[sub])]
    b = [torch.tensor(z, dtype=torch.float64, device="cuda", requires_grad=True) for z in (pts[sub], fe[sub])]
    wt = torch.as_tensor(w[sub]).cuda()
    (stokes_regvel(a[0], a[1], a[0]) * wt).sum().backward()
    (regvel_torch(torch, b[0], b[1], b[0]) * wt).sum().backward()
    res["vs_torch_autograd_direct_subset"] = {
        "points": len(sub),
        "rel_l2_d_dx": float(torch.linalg.norm(a[0].grad - b[0].grad) / torch.linalg.norm(b[0].grad)),
        "rel_l2_d_df_deps": float(torch.linalg.norm(a[1].grad - b[1].grad) / torch.linalg.norm(b[1].grad))}


def wall_inputs(cfg, seed):
    rng = np.random.default_rng(seed)
    n = cfg["n"]
    c = rng.uniform(0.1, 0.9, size=(64, 3))
    pts = c[rng.integers(0, 64, size=n)] + rng.normal(0.0, 0.02, size=(n, 3))
    pts = np.clip(pts, 0.0, 0.999)
    pts[:, 2] = 0.01 + 0.48 * pts[:, 2]
    f = rng.normal(size=(n, 3))
    if cfg["kernel"] == 16:
        f = np.concatenate([f, rng.uniform(1e-4, 5e-4, (n, 1))], axis=1)
    return pts, f


def time_wall_fmm(cfg, seed, steps, warmup, ws, flush, nsample=1000):
    """StkWallFMM_evaluate_fmm_device of one wall workload, FP64 and mixed, CUDA events per
    evaluation; accuracy against the oracle's image system on a target sample."""
    import torch
    import stkfmm_b200 as S
    pts, val = wall_inputs(cfg, seed)
    K = cfg["kernel"]
    td = S.get_kernel_dimension(K)[2]
    fmm = S.StkWallFMM(cfg["p"], cfg["max_pts"], cfg["pbc"], K)
    fmm.set_box(np.zeros(3), 1.0)
    fmm.set_points(pts, pts, None)
    t0 = time.perf_counter()
    fmm.setup_tree(K)
    res = {"workload": cfg["workload"], "setup_tree_s": time.perf_counter() - t0}
    d_v = torch.as_tensor(val).cuda()
    outs = {}
    for prec, nm in ((S.PRECISION.FP64, "fp64"), (S.PRECISION.MIXED, "mixed")):
        fmm.set_precision(prec)
        out = torch.zeros((len(pts), td), dtype=torch.float64, device="cuda")
        for _ in range(warmup):
            fmm.evaluate_fmm_device(K, d_v.data_ptr(), out.data_ptr(), None)
        torch.cuda.synchronize()
        ms = []
        torch.cuda.profiler.start()
        for _ in range(steps):
            flush.zero_()
            out.zero_()
            torch.cuda.synchronize()
            fmm.evaluate_fmm_device(K, d_v.data_ptr(), out.data_ptr(), None)
            torch.cuda.synchronize()
            ms.append(fmm.last_kernel_ms())
        torch.cuda.profiler.stop()
        m = max_over_ranks([sum(ms) / steps], ws)[0]
        res[nm] = {"evals_per_s": job_rate(1, ws, m * 1e-3), "ms_per_eval": m}
        outs[nm] = out.cpu().numpy()
    res["mixed_over_fp64"] = res["fp64"]["ms_per_eval"] / res["mixed"]["ms_per_eval"]
    res["rel_l2_mixed_vs_fp64"] = float(np.linalg.norm(outs["mixed"] - outs["fp64"]) / np.linalg.norm(outs["fp64"]))
    res["gpu_launches_per_eval"] = fmm.last_launch_count(K)
    res["timing"] = "device time of each evaluate_fmm_device (CUDA events on the wall's stream), L2 flushed between"
    res["_acc"] = (pts, val, outs, nsample)
    return res


def wall_accuracy(cfg, res):
    """Both precisions against the oracle's image system (oracle.wall_stokes / wall_rpy) on a target sample."""
    from oracle import oracle as O
    O.build()
    pts, val, outs, nsample = res.pop("_acc")
    samp = np.random.default_rng(17).choice(len(pts), nsample, replace=False)
    t0 = time.perf_counter()
    fn = O.wall_stokes if cfg["kernel"] == 8 else O.wall_rpy
    ref = fn(pts, val, pts[samp])
    res["rel_l2_vs_image_system_sample_per_component"] = {
        nm: [float(np.linalg.norm(o[samp, c] - ref[:, c]) / np.linalg.norm(ref[:, c])) for c in range(ref.shape[1])]
        for nm, o in outs.items()}
    res["sample"] = "%d targets drawn with seed 17; oracle image system over all %d sources (%.1f s on the host)" % (
        nsample, len(pts), time.perf_counter() - t0)


def run_one_workload(name, steps, warmup):
    """One further FMM or wall workload alone (for profiling); prints its block as one JSON line."""
    import torch
    torch.cuda.set_device(0)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    for cfg in EXTRA_FMM:
        if cfg["name"] == name:
            r, _, _, _ = time_extra_fmm(cfg, 0, steps, warmup, 1, flush)
            print(json.dumps({name: r}), flush=True)
            return 0
    for cfg in WALL_FMM:
        if cfg["name"] == name:
            r = time_wall_fmm(cfg, 0, steps, warmup, 1, flush)
            r.pop("_acc")
            print(json.dumps({name: r}), flush=True)
            return 0
    if name == MAIN_FMM_NAME:
        print(json.dumps({name: time_main_fmm(steps, warmup, flush)}), flush=True)
        return 0
    if name == ADJ["name"]:
        r = time_adjoint(steps, warmup, 0, 1, flush)
        adjoint_checks(r)
        print(json.dumps({name: r}), flush=True)
        return 0
    raise SystemExit("unknown workload %s" % name)


MAIN_FMM_NAME = "lappgrad_1m_clustered"


def time_main_fmm(steps, warmup, flush):
    """The headline workload's whole evaluate_fmm alone (FP64, then mixed): CUDA events
    around each evaluate_fmm_device, L2 flushed between, per-phase split; timed steps
    inside torch.cuda.profiler.start/stop."""
    import torch
    import stkfmm_b200 as S
    K = KERNEL_LAPPGRAD
    pts, q, d = make_points(0)
    fmm = S.Stk3DFMM(MULT_ORDER, MAX_PTS, S.PAXIS.NONE, K)
    fmm.set_box(np.zeros(3), 1.0)
    fmm.set_points(pts, pts, pts)
    fmm.setup_tree(K)
    stream = torch.cuda.Stream()
    qd, dd = torch.as_tensor(q).cuda(), torch.as_tensor(d).cuda()
    out = torch.zeros((N_POINTS, 4), dtype=torch.float64, device="cuda")
    res = {"workload": WORKLOAD_FMM}
    for prec, nm in ((S.PRECISION.FP64, "fp64"), (S.PRECISION.MIXED, "mixed")):
        fmm.set_precision(prec)
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                fmm.evaluate_fmm_device(K, qd.data_ptr(), out.data_ptr(), dd.data_ptr(), stream.cuda_stream)
        stream.synchronize()
        ms, phases = [], []
        torch.cuda.profiler.start()
        with torch.cuda.stream(stream):
            for _ in range(steps):
                flush.zero_()
                out.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fmm.evaluate_fmm_device(K, qd.data_ptr(), out.data_ptr(), dd.data_ptr(), stream.cuda_stream)
                e1.record(stream)
                stream.synchronize()
                ms.append(e0.elapsed_time(e1))
                phases.append(fmm.last_phase_ms(K))
        torch.cuda.profiler.stop()
        res[nm] = {"evals_per_s": 1e3 / (sum(ms) / steps), "ms_per_eval": sum(ms) / steps,
                   "phases_ms": {k: sum(p[k] for p in phases) / steps for k in phases[0]}}
    res["mixed_over_fp64"] = res["fp64"]["ms_per_eval"] / res["mixed"]["ms_per_eval"]
    return res


def run_p2p_only(steps, warmup):
    """The headline U-list P2P step alone, FP64 then mixed (for kernel profiles): `warmup`
    untimed launches then `steps` timed ones per precision, one list_p2p_kernel launch each,
    L2 flushed between timed steps; prints per-precision kernel times as one JSON line."""
    import torch
    import stkfmm_b200 as S
    torch.cuda.set_device(0)
    K = KERNEL_LAPPGRAD
    pts, q, d = make_points(0)
    fmm = S.Stk3DFMM(MULT_ORDER, MAX_PTS, S.PAXIS.NONE, K)
    fmm.set_box(np.zeros(3), 1.0)
    fmm.set_points(pts, pts, pts)
    fmm.setup_tree(K)
    st = fmm.tree_stats(K)
    stream = torch.cuda.Stream()
    qd, dd = torch.as_tensor(q).cuda(), torch.as_tensor(d).cuda()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    out = torch.zeros((N_POINTS, 4), dtype=torch.float64, device="cuda")
    res = {"workload": WORKLOAD, "point_pairs_per_step": st["u_pairs_sl"]}
    for prec, nm in ((S.PRECISION.FP64, "fp64"), (S.PRECISION.MIXED, "mixed")):
        fmm.set_precision(prec)
        kern = []
        with torch.cuda.stream(stream):
            for i in range(warmup + steps):
                flush.zero_()
                out.zero_()
                fmm.evaluate_near_device(K, qd.data_ptr(), out.data_ptr(), dd.data_ptr(), stream.cuda_stream)
                stream.synchronize()
                if i >= warmup:
                    kern.append(fmm.last_kernel_ms(K))
        res[nm] = {"kernel_ms_median": statistics.median(kern), "kernel_ms": kern}
    print(json.dumps({"p2p_only": res}), flush=True)
    return 0


def extra_fmm_inputs(cfg, seed):
    """Points, SL values and DL values (or None) of a further workload."""
    rng = np.random.default_rng(seed)
    n = cfg["n"]
    if cfg["kernel"] == 128:
        # points on sphere surfaces; SL (f, trD = 0) and DL D neutralised as Test/Test.cpp:364-402
        nsph, per = 4096, n // 4096
        centres = np.concatenate([rng.uniform(0.05, 0.95, (nsph, 2)), rng.uniform(0.05, 0.5, (nsph, 1))], axis=1)
        u = rng.normal(size=(nsph, per, 3))
        u /= np.linalg.norm(u, axis=2, keepdims=True)
        pts = (centres[:, None, :] + 0.01 * u).reshape(-1, 3)
        f = np.concatenate([rng.normal(size=(n, 3)), np.zeros((n, 1))], axis=1)
        f -= f.mean(0)
        d = rng.normal(size=(n, 9))
        tr = (d[:, 0] + d[:, 4] + d[:, 8]).mean() / 3
        d[:, [0, 4, 8]] -= tr
        return pts, f, d
    pts = rng.random((n, 3))
    f = rng.normal(size=(n, 3))
    if cfg["pbc"]:
        f -= f.mean(0)  # net force removed for the periodic sum (Test/Test.cpp:332-351)
    if cfg["kernel"] == 16:
        f = np.concatenate([f, rng.uniform(1e-4, 5e-4, (n, 1))], axis=1)
    return pts, f, None


def time_extra_fmm(cfg, seed, steps, warmup, ws, flush):
    """evaluate_fmm_device of one further workload, FP64 and mixed, CUDA events per evaluation."""
    import torch
    import stkfmm_b200 as S
    pts, slv, dlv = extra_fmm_inputs(cfg, seed)
    K = cfg["kernel"]
    td = S.get_kernel_dimension(K)[2]
    fmm = S.Stk3DFMM(cfg["p"], cfg["max_pts"], cfg["pbc"], K)
    fmm.set_box(np.zeros(3), 1.0)
    fmm.set_points(pts, pts, pts if dlv is not None else None)
    t0 = time.perf_counter()
    fmm.setup_tree(K)
    tree_s = time.perf_counter() - t0
    d_sl = torch.as_tensor(slv).cuda()
    d_dl = torch.as_tensor(dlv).cuda() if dlv is not None else None
    dlp = d_dl.data_ptr() if d_dl is not None else 0
    res = {"workload": cfg["workload"], "tree": fmm.tree_stats(K), "setup_tree_s": tree_s}
    outs = {}
    for prec, nm in ((S.PRECISION.FP64, "fp64"), (S.PRECISION.MIXED, "mixed")):
        fmm.set_precision(prec)
        out = torch.zeros((len(pts), td), dtype=torch.float64, device="cuda")
        t0 = time.perf_counter()
        for _ in range(warmup):
            fmm.evaluate_fmm_device(K, d_sl.data_ptr(), out.data_ptr(), dlp, None)
        torch.cuda.synchronize()
        if nm == "fp64":
            res["first_evaluations_s"] = time.perf_counter() - t0  # includes the far-field operator build
        ms, phases = [], []
        torch.cuda.profiler.start()
        for _ in range(steps):
            flush.zero_()
            out.zero_()
            torch.cuda.synchronize()
            fmm.evaluate_fmm_device(K, d_sl.data_ptr(), out.data_ptr(), dlp, None)
            torch.cuda.synchronize()
            ms.append(fmm.last_kernel_ms(K))
            phases.append(fmm.last_phase_ms(K))
        torch.cuda.profiler.stop()
        m = max_over_ranks([sum(ms) / steps], ws)[0]
        res[nm] = {"evals_per_s": job_rate(1, ws, m * 1e-3), "ms_per_eval": m,
                   "phases_ms": {k: sum(p[k] for p in phases) / steps for k in phases[0]}}
        outs[nm] = out.cpu().numpy()
    res["mixed_over_fp64"] = res["fp64"]["ms_per_eval"] / res["mixed"]["ms_per_eval"]
    res["rel_l2_mixed_vs_fp64"] = float(np.linalg.norm(outs["mixed"] - outs["fp64"]) / np.linalg.norm(outs["fp64"]))
    res["work_per_eval"] = fmm.fmm_stats(K)
    res["m2l_roofline"] = m2l_roofline(fmm, K, res)
    res["gpu_launches_per_eval"] = fmm.last_launch_count(K)
    res["timing"] = "device time of each evaluate_fmm_device (CUDA events on the handle's stream), L2 flushed between"
    if cfg["pbc"]:
        res["convergence_vs_p%d" % (cfg["p"] + 2)] = periodic_convergence(cfg, K, pts, slv, dlv, d_sl, dlp, outs)
    return res, pts, slv, outs


def periodic_convergence(cfg, K, pts, slv, dlv, d_sl, dlp, outs):
    """Accuracy of a periodic workload at full size by the reference's own protocol for periodic
    boxes (Test/Test.cpp's errorConvergence: the FMM against the same FMM at a higher order; the
    reference's periodic tests check convergence and translation, not an Ewald sum): both
    precisions against FP64 at p + 2, relative L2 per output component, as is and with the mean
    difference (the reference's "drift", Test/Test.cpp:143-150) removed."""
    import torch
    import stkfmm_b200 as S
    pc = cfg["p"] + 2
    td = S.get_kernel_dimension(K)[2]
    f = S.Stk3DFMM(pc, cfg["max_pts"], cfg["pbc"], K)
    f.set_box(np.zeros(3), 1.0)
    f.set_points(pts, pts, pts if dlv is not None else None)
    f.setup_tree(K)
    t0 = time.perf_counter()
    out = torch.zeros((len(pts), td), dtype=torch.float64, device="cuda")
    f.evaluate_fmm_device(K, d_sl.data_ptr(), out.data_ptr(), dlp, None)
    torch.cuda.synchronize()
    ref = out.cpu().numpy()
    # the U-list near field alone (the same lists at both orders, evaluated exactly by both):
    # ref - near is the part the far field approximates, the denominator of far_part errors
    out.zero_()
    f.set_precision(S.PRECISION.FP64)
    f.evaluate_near_device(K, d_sl.data_ptr(), out.data_ptr(), dlp, None)
    torch.cuda.synchronize()
    far = ref - out.cpu().numpy()
    res = {"reference": "FP64 FMM at p = %d, same points and tree rules (%.1f s incl. its operator build)"
                        % (pc, time.perf_counter() - t0),
           "far_part": "rel_l2_vs_far_part_per_component divides by the norm of the reference minus its U-list "
                       "near field (the part the far field approximates); on points whose nearest neighbours "
                       "are very close the whole-output norm is set by exact near pairs"}
    for nm, o in outs.items():
        d = o - ref
        res[nm] = {"rel_l2_per_component": [float(np.linalg.norm(d[:, c]) / np.linalg.norm(ref[:, c]))
                                            for c in range(td)],
                   "rel_l2_vs_far_part_per_component": [float(np.linalg.norm(d[:, c]) / np.linalg.norm(far[:, c]))
                                                        for c in range(td)],
                   "rel_l2_drift_removed_per_component": [
                       float(np.linalg.norm(d[:, c] - d[:, c].mean()) / np.linalg.norm(ref[:, c] - ref[:, c].mean()))
                       for c in range(td)],
                   "drift_per_component": [float(d[:, c].mean()) for c in range(td)]}
    del f
    return res


def m2l_roofline(fmm, K, res):
    """Achieved FP64 / FP32 rate of the compressed M2L phase (its flops over its event time)."""
    w = fmm.m2l_work(K)
    out = {"flops_algorithmic": w["flops_algorithmic"], "flops_executed": w["flops_executed"]}
    for nm in ("fp64", "mixed"):
        ms = res[nm]["phases_ms"]["m2l"] if nm in res else None
        if ms:
            out[nm + "_tflops_algorithmic"] = w["flops_algorithmic"] / (ms * 1e-3) / 1e12
            out[nm + "_tflops_executed"] = w["flops_executed"] / (ms * 1e-3) / 1e12
    out["note"] = ("M2L phase: basis products, column gather, per-offset GEMMs, per-target reduce; "
                   "FP64 GEMMs on the FP64 tensor pipe (DMMA), mixed GEMMs on the tcgen05 tensor cores (3xTF32), basis products FP64")
    return out


def extra_fmm_accuracy(cfg, pts, slv, outs, nsample=4096):
    """Free-space workloads: both precisions against the oracle's direct sum on a target sample.
    The RPY PXYZ workload: against its Ewald-summed fixture (tests/golden/rpy_pxyz_2m_ewald.npz,
    4,096 sampled targets, made by tests/golden/make_rpy_pxyz_ewald.py)."""
    if cfg["pbc"]:
        fx = os.path.join(ROOT, "tests", "golden", "rpy_pxyz_2m_ewald.npz")
        if cfg["name"] != "rpy_pxyz_2m_uniform" or not os.path.exists(fx):
            return None
        z = np.load(fx)
        idx, ref = z["idx"], z["truth"]
        return {nm: [float(np.linalg.norm(o[idx, c] - ref[:, c]) / np.linalg.norm(ref[:, c]))
                     for c in range(ref.shape[1])] for nm, o in outs.items()}
    from oracle import oracle as O
    O.build()
    samp = np.random.default_rng(13).choice(len(pts), min(nsample, len(pts)), replace=False)
    uk = {8: O.UK_STOKES_VEL}[cfg["kernel"]]
    ref = O.direct(uk, pts, slv, pts[samp])
    return {nm: [float(np.linalg.norm(o[samp, c] - ref[:, c]) / np.linalg.norm(ref[:, c]))
                 for c in range(ref.shape[1])] for nm, o in outs.items()}


def time_fmm_sharded(steps, warmup, ws, rank, stream, flush):
    """Multi-GPU (ws > 1): ONE LapPGrad FMM problem (the seed-0 points on every rank) split over
    the ranks -- near field, L2T and M2T by work items (set_shard), M2L / S2L by target node with
    one NCCL all-reduce of the downward densities per evaluation (set_allreduce) -- timed with CUDA
    events, max over ranks (strong scaling).  Returns the block and the all-reduced output."""
    import torch
    import torch.distributed as dist
    import stkfmm_b200 as S
    from stkfmm_b200.stkfmm import torch_allreduce
    K = KERNEL_LAPPGRAD
    pts, q, d = make_points(0)
    fmm = S.Stk3DFMM(MULT_ORDER, MAX_PTS, S.PAXIS.NONE, K)
    fmm.set_box(np.zeros(3), 1.0)
    fmm.set_points(pts, pts, pts)
    fmm.set_shard(rank, ws)
    fmm.set_allreduce(torch_allreduce())
    fmm.setup_tree(K)
    qd, dd = torch.as_tensor(q).cuda(), torch.as_tensor(d).cuda()
    sp = stream.cuda_stream
    out = torch.zeros((N_POINTS, 4), dtype=torch.float64, device="cuda")
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            out.zero_()
            fmm.evaluate_fmm_device(K, qd.data_ptr(), out.data_ptr(), dd.data_ptr(), sp)
    stream.synchronize()
    ms = []
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            out.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fmm.evaluate_fmm_device(K, qd.data_ptr(), out.data_ptr(), dd.data_ptr(), sp)
            e1.record(stream)
        stream.synchronize()
        ms.append(e0.elapsed_time(e1))
    m = max_over_ranks([sum(ms) / len(ms)], ws)[0]
    total = out.clone()
    dist.all_reduce(total)
    block = {"workload": WORKLOAD_FMM + "; one problem split over %d GPUs" % ws, "ranks": ws,
             "evals_per_s": 1e3 / m, "ms_per_eval": m, "scaling": "strong",
             "split": "near field / L2T / M2T by cost-dealt work items; M2L / S2L by target node; one NCCL "
                      "all-reduce of the downward equivalent densities per evaluation",
             "timing": "CUDA events on the evaluation stream, max over ranks, L2 flushed between"}
    return block, total


# ---------------------------------------------------------- CPU baseline ----
def sample_boxes(ul, budget_pairs, seed=1):
    """Random target leaves of the U-list whose SL+DL pairs sum to ~budget_pairs."""
    tb, te, off, ent = ul["trg_begin"], ul["trg_end"], ul["list_off"], ul["list_ent"]
    sb, se = ul["sl_begin"], ul["sl_end"]
    cnt = se - sb
    nt = te - tb
    ns = np.array([cnt[ent[off[b]:off[b + 1]] >> 5].sum() for b in range(len(tb))], dtype=np.int64)
    cand = np.flatnonzero((nt > 0) & (ns > 0))
    rng = np.random.default_rng(seed)
    rng.shuffle(cand)
    pick, tot = [], 0
    for b in cand:
        pick.append(b)
        tot += 2 * int(nt[b]) * int(ns[b])
        if tot >= budget_pairs:
            break
    pick = np.array(sorted(pick), dtype=np.int64)
    return pick, tot


def cpu_lists_prepare(ul, pts, q, d, boxes):
    """The sampled U-list boxes in the CSR form the CPU kernels take, with the
    points, values and output in leaf order (set-up, not timed: the reference
    keeps its points in tree order inside PVFMM)."""
    tb, te, off, ent = ul["trg_begin"][boxes], ul["trg_end"][boxes], ul["list_off"], ul["list_ent"]
    noff = np.zeros(len(boxes) + 1, np.int64)
    ents = []
    for i, b in enumerate(boxes):
        e = ent[off[b]:off[b + 1]]
        ents.append(e)
        noff[i + 1] = noff[i] + len(e)
    ents = np.concatenate(ents) if ents else np.zeros(0, np.int32)
    sp, tp = ul["sl_perm"], ul["trg_perm"]
    as_i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    return {"tb": as_i32(tb), "te": as_i32(te), "off": as_i32(noff), "src_box": as_i32(ents >> 5),
            "shift": as_i32(ents & 31), "sl_b": as_i32(ul["sl_begin"]), "sl_e": as_i32(ul["sl_end"]),
            "dl_b": as_i32(ul["dl_begin"]), "dl_e": as_i32(ul["dl_end"]),
            "src": np.ascontiguousarray(pts[sp]), "trg": np.ascontiguousarray(pts[tp]),
            "q": np.ascontiguousarray(q[sp]), "d": np.ascontiguousarray(d[sp]), "out": np.zeros((len(pts), 4))}


def cpu_lists_run(w, use_ref):
    """The reference's kernels (oracle/_ref, SimpleKernel) or the oracle port over
    the prepared U-list boxes; adds into w["out"]."""
    from oracle import oracle as O
    if use_ref:
        O.ref_lists(O.REF_LAP_SL_PGRAD, w["tb"], w["te"], w["off"], w["src_box"], w["sl_b"], w["sl_e"], w["src"],
                    w["q"], w["trg"], out=w["out"])
        O.ref_lists(O.REF_LAP_DL_PGRAD, w["tb"], w["te"], w["off"], w["src_box"], w["dl_b"], w["dl_e"], w["src"],
                    w["d"], w["trg"], out=w["out"])
    else:
        O.lists(O.UK_LAPLACE_PGRAD, w["tb"], w["te"], w["off"], w["src_box"], w["shift"], w["sl_b"], w["sl_e"],
                w["src"], w["q"], w["trg"], out=w["out"])
        O.lists(O.UK_LAPLACE_DIPOLEPGRAD, w["tb"], w["te"], w["off"], w["src_box"], w["shift"], w["dl_b"], w["dl_e"],
                w["src"], w["d"], w["trg"], out=w["out"])
    return w["out"]


def host_ulist(pts):
    """The benchmark's U list, built by the host-only tree library (libstk_octree.so: no GPU
    library is loaded); the same tree, lists and leaf order as the GPU handle's setup_tree.
    Target ranges of internal nodes are emptied (U lists belong to leaves)."""
    import stkfmm_b200 as S
    t = S.Octree(pts, MAX_PTS, 0, sl=pts, dl=pts, trg=pts)
    ul = {}
    ul["list_off"], ul["list_ent"] = t.list("U")
    leaf = t.first_child < 0
    for k, nm in enumerate(("sl", "dl", "trg")):
        perm, b, e = t.point_set(k)
        ul[nm + "_perm"] = perm
        if nm == "trg":
            e = np.where(leaf, e, b)
        ul[nm + "_begin"], ul[nm + "_end"] = b, e
    return ul


def ulist_pairs(ul):
    """Exact (target, source point) pairs of the U list (SL; DL is the same at the same points)."""
    off, ent = ul["list_off"], ul["list_ent"]
    cnt = (ul["sl_end"] - ul["sl_begin"]).astype(np.int64)
    per_entry = cnt[ent >> 5]
    csum = np.concatenate([[0], np.cumsum(per_entry)])
    ns = csum[off[1:]] - csum[off[:-1]]
    nt = (ul["trg_end"] - ul["trg_begin"]).astype(np.int64)
    return int((nt * ns).sum())


def cpu_full_prepare(ul, pts, q, d):
    """The whole U list in the form the SIMD reference loop takes: leaf-ordered points and
    values, list arrays (set-up, not timed: the reference keeps its points in tree order
    inside PVFMM)."""
    sp, tp = ul["sl_perm"], ul["trg_perm"]
    as_i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    ent = ul["list_ent"]
    return {"tb": as_i32(ul["trg_begin"]), "te": as_i32(ul["trg_end"]), "off": as_i32(ul["list_off"]),
            "src_box": as_i32(ent >> 5), "shift": as_i32(ent & 31), "sl_b": as_i32(ul["sl_begin"]),
            "sl_e": as_i32(ul["sl_end"]), "dl_b": as_i32(ul["dl_begin"]), "dl_e": as_i32(ul["dl_end"]),
            "src": np.ascontiguousarray(pts[sp]), "trg": np.ascontiguousarray(pts[tp]),
            "q": np.ascontiguousarray(q[sp]), "d": np.ascontiguousarray(d[ul["dl_perm"]]),
            "out": np.zeros((len(pts), 4))}


def cpu_full_step(w, nthreads=0):
    """One full step on the host: the reference's laplace_pgrad and laplace_dipolepgrad
    bodies over the whole U list (PVFMM-style SIMD loop, OpenMP over target leaves)."""
    from oracle import oracle as O
    O.ref_simd_lists(O.REF_SIMD_LAP_PGRAD, w["tb"], w["te"], w["off"], w["src_box"], w["shift"], w["sl_b"],
                     w["sl_e"], w["src"], w["q"], w["trg"], out=w["out"], nthreads=nthreads)
    O.ref_simd_lists(O.REF_SIMD_LAP_DIPOLEPGRAD, w["tb"], w["te"], w["off"], w["src_box"], w["shift"], w["dl_b"],
                     w["dl_e"], w["src"], w["d"], w["trg"], out=w["out"], nthreads=nthreads)
    return w["out"]


def cpu_isa():
    from oracle import oracle as O
    return os.path.basename(O.ref_simd_path())


def cpu_baseline(ul, pts, q, d, pairs, target_seconds=15.0):
    """The reference's micro-kernels in PVFMM's SIMD loop over the whole step's U list, full
    steps on all host cores; the reference's scalar test kernel (SimpleKernel) beside it on a
    bounded sample."""
    from oracle import oracle as O
    O.build()
    cores = os.cpu_count() or 1
    w = cpu_full_prepare(ul, pts, q, d)
    cpu_full_step(w)  # thread pool and pages warm
    t0 = time.perf_counter()
    cpu_full_step(w)
    one = time.perf_counter() - t0
    reps = int(max(1, min(10, target_seconds / max(one, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(reps):
        cpu_full_step(w)
    dt = (time.perf_counter() - t0) / reps
    out = {"value": pairs / dt, "unit": "pairs/s", "cores": cores, "kind": "reference",
           "sample": "the whole step (%.4g SL+DL pairs), %d repeats: the reference's laplace_pgrad + "
                     "laplace_dipolepgrad uKerEval bodies (Lib/include/STKFMM/LaplaceLayerKernel.hpp, compiled in "
                     "place) in a PVFMM-style SIMD pair loop (%s, OpenMP %d threads), FP64"
                     % (pairs, reps, cpu_isa(), cores),
           "ms_per_step": dt * 1e3}
    if O.ref_available():
        boxes, spairs = sample_boxes(ul, 2e8, seed=2)
        ws = cpu_lists_prepare(ul, pts, q, d, boxes)
        t0 = time.perf_counter()
        cpu_lists_run(ws, True)
        sdt = time.perf_counter() - t0
        out["simple_kernel"] = {"value": spairs / sdt, "unit": "pairs/s", "cores": cores,
                                "sample": "the reference's scalar test kernels Test/SimpleKernel.cpp LaplaceSLPGrad + "
                                          "LaplaceDLPGrad over the U lists of %d random target leaves (%.3g pairs)"
                                          % (len(boxes), spairs)}
    return out


# ---------------------------------------------------------------- arms ------
def reference_arm(args):
    """The reference's CPU implementation of the step (its micro-kernel bodies in PVFMM's SIMD
    loop, all host cores) on the same config: each step is the whole U-list pass."""
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    from oracle import oracle as O
    O.build()
    if not O.ref_simd_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built (reference tree absent "
                                                              "where the library was built)"}), flush=True)
        return 0
    pts, q, d = make_points(0)
    ul = host_ulist(pts)
    pairs = 2 * ulist_pairs(ul)
    w = cpu_full_prepare(ul, pts, q, d)
    for _ in range(args.warmup):
        cpu_full_step(w)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        cpu_full_step(w)
        times.append(time.perf_counter() - t0)
    dt = sum(times) / len(times)
    value = pairs / dt
    cores = os.cpu_count() or 1
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n_points": N_POINTS, "pairs_per_step": pairs, "same_config": True,
                       "step": "the whole U-list S2T pass (SL + DL), as the GPU arm's step"},
            "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": cores, "kind": "reference",
                             "sample": "the whole step: the reference's laplace_pgrad + laplace_dipolepgrad uKerEval "
                                       "bodies (LaplaceLayerKernel.hpp, compiled in place) in a PVFMM-style SIMD pair "
                                       "loop (%s), OpenMP %d threads, FP64" % (cpu_isa(), cores)},
            "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def b200_arm(args):
    import torch
    import torch.distributed as dist

    ws, rank, local = dist_env()
    if ws > 1:
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    import stkfmm_b200 as S
    from stkfmm_b200._lib import lib

    K = KERNEL_LAPPGRAD
    pts, q, d = make_points(rank)
    fmm = S.Stk3DFMM(MULT_ORDER, MAX_PTS, S.PAXIS.NONE, K)
    fmm.set_box(np.zeros(3), 1.0)
    fmm.set_points(pts, pts, pts)
    t0 = time.perf_counter()
    fmm.setup_tree(K)
    tree_s = time.perf_counter() - t0
    st = fmm.tree_stats(K)
    pairs = st["u_pairs_sl"] + st["u_pairs_dl"]
    point_pairs = st["u_pairs_sl"]

    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    qd = torch.as_tensor(q).cuda()
    dd = torch.as_tensor(d).cuda()
    outs = {}
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def barrier():
        if ws > 1:
            dist.barrier()

    def run(prec, steps, warmup):
        fmm.set_precision(prec)
        out = torch.zeros((N_POINTS, 4), dtype=torch.float64, device="cuda")
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                fmm.evaluate_near_device(K, qd.data_ptr(), out.data_ptr(), dd.data_ptr(), sp)
        stream.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        kern = []
        barrier()
        torch.cuda.synchronize()
        tw0 = time.perf_counter()
        torch.cuda.profiler.start()  # a profiler started with --profile-from-start off sees only timed steps
        with torch.cuda.stream(stream):
            for i in range(steps):
                flush.zero_()  # L2 flush (256 MB write) between timed steps, outside the step events
                out.zero_()
                evs[i][0].record(stream)
                fmm.evaluate_near_device(K, qd.data_ptr(), out.data_ptr(), dd.data_ptr(), sp)
                evs[i][1].record(stream)
                stream.synchronize()
                kern.append(fmm.last_kernel_ms(K))
        torch.cuda.profiler.stop()
        torch.cuda.synchronize()
        barrier()
        wall = time.perf_counter() - tw0
        step_ms = [a.elapsed_time(b) for a, b in evs]
        ms = sum(step_ms) / len(step_ms)
        kms = sum(kern) / len(kern)
        ms, kms = max_over_ranks([ms, kms], ws)
        outs[prec] = out
        return ms, kms, wall

    def run_fmm(prec, steps, warmup):
        """Whole evaluate_fmm (near field + KIFMM far field) on device-resident values."""
        fmm.set_precision(prec)
        out = torch.zeros((N_POINTS, 4), dtype=torch.float64, device="cuda")
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                fmm.evaluate_fmm_device(K, qd.data_ptr(), out.data_ptr(), dd.data_ptr(), sp)
        stream.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        phases = []
        barrier()
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        with torch.cuda.stream(stream):
            for i in range(steps):
                flush.zero_()
                out.zero_()
                evs[i][0].record(stream)
                fmm.evaluate_fmm_device(K, qd.data_ptr(), out.data_ptr(), dd.data_ptr(), sp)
                evs[i][1].record(stream)
                stream.synchronize()
                phases.append(fmm.last_phase_ms(K))
        torch.cuda.profiler.stop()
        torch.cuda.synchronize()
        barrier()
        ms = max_over_ranks([sum(a.elapsed_time(b) for a, b in evs) / steps], ws)[0]
        ph = {k: sum(p[k] for p in phases) / steps for k in phases[0]}
        return ms, ph, out

    clocks = ClockSampler(dev) if rank == 0 else None
    if clocks:
        clocks.start()
    ms64, k64, _ = run(S.PRECISION.FP64, args.steps, args.warmup)
    near_launches = fmm.last_launch_count(K)
    msmx, kmx, _ = run(S.PRECISION.MIXED, args.steps, args.warmup)
    fms64, fph64, fout64 = run_fmm(S.PRECISION.FP64, args.steps, args.warmup)
    fmsmx, fphmx, foutmx = run_fmm(S.PRECISION.MIXED, args.steps, args.warmup)
    fmm_launches = fmm.last_launch_count(K)
    fst = fmm.fmm_stats(K)
    clk = clocks.stop() if clocks else None

    value = job_rate(pairs, ws, ms64 * 1e-3)  # the headline: FP64, the reference's precision
    value_mx = job_rate(pairs, ws, msmx * 1e-3)
    o64 = outs[S.PRECISION.FP64].double()
    omx = outs[S.PRECISION.MIXED].double()
    err_mx = float(torch.linalg.norm(omx - o64) / torch.linalg.norm(o64))
    err_cols = [float(torch.linalg.norm(omx[:, c] - o64[:, c]) / torch.linalg.norm(o64[:, c])) for c in range(4)]

    # ---- e2e: the C-ABI host call (pinned host buffers in and out, copies inside), both paths ----
    qh = torch.as_tensor(q).pin_memory().numpy()
    dh = torch.as_tensor(d).pin_memory().numpy()
    oh = torch.zeros((N_POINTS, 4), dtype=torch.float64).pin_memory().numpy()

    def e2e_near(prec):
        fmm.set_precision(prec)
        for _ in range(args.warmup):
            fmm.evaluate_near(K, qh, oh, dh)
        barrier()
        tt = []
        for _ in range(args.steps):
            oh[:] = 0.0
            t0 = time.perf_counter()
            fmm.evaluate_near(K, qh, oh, dh)
            tt.append(time.perf_counter() - t0)
        return max_over_ranks([sum(tt) / len(tt)], ws)[0]

    e2e_s = e2e_near(S.PRECISION.FP64)
    e2e_val = job_rate(pairs, ws, e2e_s)
    e2e_mx_s = e2e_near(S.PRECISION.MIXED)

    # ---- FMM e2e: Stk3DFMM_evaluate_fmm with pinned host arrays (FP64) ----
    fmm.set_precision(S.PRECISION.FP64)
    for _ in range(args.warmup):
        fmm.evaluate_fmm(K, qh, oh, dh)
    barrier()
    fe2e_t = []
    for _ in range(args.steps):
        oh[:] = 0.0
        t0 = time.perf_counter()
        fmm.evaluate_fmm(K, qh, oh, dh)
        fe2e_t.append(time.perf_counter() - t0)
    fe2e_s = max_over_ranks([sum(fe2e_t) / len(fe2e_t)], ws)[0]

    # ---- the further FMM workloads (configs 1 and 3): every rank runs its own replica ----
    extra = []
    for cfg in EXTRA_FMM:
        # a few timed evaluations each (the largest takes about a second per evaluation)
        r, epts, eslv, eouts = time_extra_fmm(cfg, rank, min(args.steps, 3), args.warmup, ws, flush)
        extra.append((cfg, r, epts, eslv, eouts))
    walls = [(cfg, time_wall_fmm(cfg, rank, min(args.steps, 3), args.warmup, ws, flush)) for cfg in WALL_FMM]
    adj = time_adjoint(min(args.steps, 5), args.warmup, rank, ws, flush)
    sharded = time_fmm_sharded(min(args.steps, 5), args.warmup, ws, rank, stream, flush) if ws > 1 else None

    # the last collective: rank 0's checks and report below are host work, so no rank
    # waits on them (they take tens of seconds, against the group's 120 s timeout)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0

    # ---- parity spot check of the timed FP64 output against the oracle ----
    ul = fmm.ulist(K)
    from oracle import oracle as O
    O.build()
    boxes, _ = sample_boxes(ul, 2e7, seed=5)
    ref_sorted = cpu_lists_run(cpu_lists_prepare(ul, pts, q, d, boxes), use_ref=False)
    sel = np.concatenate([np.arange(ul["trg_begin"][b], ul["trg_end"][b]) for b in boxes])
    gpu64 = o64.cpu().numpy()[ul["trg_perm"][sel]]
    parity64 = float(np.linalg.norm(gpu64 - ref_sorted[sel]) / np.linalg.norm(ref_sorted[sel]))

    # ---- roofline of the dominant kernel (the fused FP64 P2P kernel of the headline) ----
    peaks = np.zeros(6)
    lib().stk_measure_peaks(peaks.ctypes.data_as(__import__("stkfmm_b200._lib", fromlist=["P_d"]).P_d))
    achieved = point_pairs * FLOPS_PER_POINT_PAIR / (k64 * 1e-3) / 1e12
    achieved_mx = point_pairs * FLOPS_PER_POINT_PAIR / (kmx * 1e-3) / 1e12
    traffic, traffic_mx = None, None
    tj = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tj):
        try:
            tt = json.load(open(tj))
            traffic = tt.get("list_p2p_kernel<LAPLACE_SLDL_PGRAD,fp64>")
            traffic_mx = tt.get("list_p2p_kernel<LAPLACE_SLDL_PGRAD,mixed>")
        except Exception:
            traffic = None

    cpu = cpu_baseline(ul, pts, q, d, pairs) if ws == 1 else None

    # ---- FMM accuracy: both precisions against the oracle's direct sum on a target sample ----
    samp = np.random.default_rng(11).choice(N_POINTS, FMM_SAMPLE, replace=False)
    t0 = time.perf_counter()
    ref = O.direct(O.UK_LAPLACE_PGRAD, pts, q, pts[samp]) + O.direct(O.UK_LAPLACE_DIPOLEPGRAD, pts, d, pts[samp])
    oracle_s = time.perf_counter() - t0
    fmm_err = {}
    for name, o in (("fp64", fout64), ("mixed", foutmx)):
        got = o.cpu().numpy()[samp]
        fmm_err[name] = {"all": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
                         "per_component": [float(np.linalg.norm(got[:, c] - ref[:, c]) / np.linalg.norm(ref[:, c]))
                                           for c in range(4)]}
    extra_blocks = {}
    for cfg, r, epts, eslv, eouts in extra:
        r["rel_l2_vs_ewald_sample_per_component" if cfg["pbc"] else "rel_l2_vs_direct_sum_sample_per_component"] = \
            extra_fmm_accuracy(cfg, epts, eslv, eouts)
        extra_blocks[cfg["name"]] = r
    for cfg, r in walls:
        wall_accuracy(cfg, r)
        extra_blocks[cfg["name"]] = r
    adjoint_checks(adj)
    if sharded is not None:
        # rank 0's own FMM leg ran the same seed-0 points unsharded
        blk, total = sharded
        blk["rel_l2_vs_unsharded_fp64"] = float(torch.linalg.norm(total - fout64) / torch.linalg.norm(fout64))
        sharded = blk
    fmm_block = {
        "workload": WORKLOAD_FMM,
        "fp64": {"evals_per_s": job_rate(1, ws, fms64 * 1e-3), "ms_per_eval": fms64, "phases_ms": fph64},
        "mixed": {"evals_per_s": job_rate(1, ws, fmsmx * 1e-3), "ms_per_eval": fmsmx, "phases_ms": fphmx},
        "mixed_over_fp64": fms64 / fmsmx,
        "rel_l2_vs_direct_sum_sample": fmm_err,
        "sample": "%d targets drawn with seed 11; oracle direct sum over all %d sources (%.1f s on the host)"
                  % (FMM_SAMPLE, N_POINTS, oracle_s),
        "work_per_eval": fst,
        "m2l_roofline": m2l_roofline(fmm, K, {"fp64": {"phases_ms": fph64}, "mixed": {"phases_ms": fphmx}}),
        "e2e": {"evals_per_s": job_rate(1, ws, fe2e_s), "ms_per_eval": fe2e_s * 1e3,
                "api": "Stk3DFMM_evaluate_fmm (C ABI, pinned host arrays, FP64)",
                "h2d_bytes_per_eval": int(q.nbytes + d.nbytes + N_POINTS * 4 * 8),
                "d2h_bytes_per_eval": int(N_POINTS * 4 * 8)},
        "gpu_launches_per_eval": fmm_launches,
        "timing": "CUDA events on the launching stream around each evaluate_fmm_device, 256 MB L2 flush between",
    }

    line = {
        "metric": METRIC,
        "value": value, "unit": "pairs/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms64, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_points": N_POINTS, "tree_nodes": st["nodes"], "leaves": st["leaves"],
                   "depth": st["depth"], "u_entries": st["u_entries"], "pairs_per_step": pairs,
                   "point_pairs_per_step": point_pairs, "l2": "256 MB write between timed steps (inputs < L2)",
                   "parallelism": "replica per GPU" if ws > 1 else "1 GPU", "setup_tree_s": tree_s},
        "fp64": {"value": value, "unit": "pairs/s", "ms_per_step": ms64, "kernel_ms": k64},
        "mixed": {"value": value_mx, "unit": "pairs/s", "ms_per_step": msmx, "kernel_ms": kmx,
                  "dtype": "f32 kernel tensor (f64 displacement split hi/lo, Kahan f32 accumulation)",
                  "e2e": {"value": job_rate(pairs, ws, e2e_mx_s), "unit": "pairs/s", "ms_per_step": e2e_mx_s * 1e3}},
        "mixed_over_fp64": value_mx / value,
        "mixed_over_fp64_kernel": k64 / kmx,
        "rel_l2_mixed_vs_fp64": err_mx, "rel_l2_mixed_vs_fp64_per_component": err_cols,
        "rel_l2_fp64_vs_oracle_sample": parity64,
        "fmm_evals_per_s": job_rate(1, ws, fms64 * 1e-3),
        "fmm": fmm_block,
        "fmm_other_workloads": extra_blocks,
        "adjoint": adj,
        "fmm_sharded": sharded,
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": float(peaks[1]), "unit": "TFLOP/s",
                     "frac": achieved / float(peaks[1]) if peaks[1] > 0 else None, "traffic": traffic,
                     "kernel": "list_p2p_kernel<LAPLACE_SLDL_PGRAD, fp64>", "kernel_ms": k64,
                     "flops_per_point_pair": FLOPS_PER_POINT_PAIR,
                     "peak_source": "measured FP64 FMA probe (stk_measure_peaks) on this GPU, of measured",
                     "probe": {"fp32_tflops": float(peaks[0]), "fp64_tflops": float(peaks[1]),
                               "mufu_rsqrt_gops": float(peaks[2]), "probe_sm_mhz": float(peaks[3]),
                               "fp32x2_tflops": float(peaks[5])},
                     "mixed_path": {"bound": "fp32", "achieved": achieved_mx, "peak": float(peaks[0]),
                                    "frac": achieved_mx / float(peaks[0]) if peaks[0] > 0 else None,
                                    "kernel": "list_p2p_kernel<LAPLACE_SLDL_PGRAD, mixed>", "kernel_ms": kmx,
                                    "traffic": traffic_mx}},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_val, "unit": "pairs/s", "h2d_bytes_per_step": int(q.nbytes + d.nbytes + N_POINTS * 4 * 8),
                "d2h_bytes_per_step": int(N_POINTS * 4 * 8), "ms_per_step": e2e_s * 1e3,
                "api": "Stk3DFMM_evaluate_near (C ABI, pinned host arrays, FP64)"},
        # own kernels launched in the timed regions: the P2P steps and FMM evaluations of both
        # precisions, the further workloads' timed evaluations, the adjoint steps (pack + list
        # kernel for the forward and each adjoint pass)
        "gpu_launches": (args.steps * (2 * near_launches + 2 * fmm_launches)
                         + sum(2 * min(args.steps, 3) * b["gpu_launches_per_eval"] for b in extra_blocks.values())
                         + 2 * min(args.steps, 5) * 6),
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--fmm-workload", default=None,
                    help="time one FMM / wall workload alone (%s) and print its block"
                         % ", ".join([MAIN_FMM_NAME] + [c["name"] for c in EXTRA_FMM + WALL_FMM] + [ADJ["name"]]))
    ap.add_argument("--p2p-only", action="store_true",
                    help="time the U-list P2P step alone, FP64 then mixed (one kernel launch per step)")
    args = ap.parse_args()
    if args.p2p_only:
        return run_p2p_only(args.steps, args.warmup)
    if args.fmm_workload:
        return run_one_workload(args.fmm_workload, args.steps, args.warmup)
    if args.impl == "reference":
        return reference_arm(args)
    return b200_arm(args)


if __name__ == "__main__":
    sys.exit(main())
