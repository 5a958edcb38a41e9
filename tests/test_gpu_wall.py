"""GPU: StkWallFMM (Stokeslets / RPY spheres above a no-slip wall) against the
oracle's restatement of the reference's image systems (oracle/oracle.py:
wall_stokes, wall_rpy, after Lib/src/StkWallFMM.cpp:154-292), which is itself
pinned by the no-slip condition (tests/test_oracle.py), and the reference's own
wall check: zero velocity on the wall (Test/Test.cpp:222-240, Test/main.cpp:32-40).
Error measure: relative L2 per output component (Test/Test.cpp:113-151).
"""
import numpy as np
import pytest

from conftest import component_errors, rel_l2
from helpers import clustered_points
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = {8: 5e-5, 10: 5e-6}


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def wall_points(rng, n, box=1.0, origin=(0.0, 0.0, 0.0)):
    """Clustered points in [0,1)^2 x [0.01, 0.49), mapped to [o, o+L)^2 x [o_z, o_z + L/2)."""
    p = np.minimum(clustered_points(rng, n, nclusters=5, sigma=0.05), 0.999)
    p[:, 2] = 0.01 + 0.48 * p[:, 2]
    return p * box + np.asarray(origin)


def run_wall(kernel, p, max_pts, pbc, src, trg, val, box=1.0, origin=(0.0, 0.0, 0.0), prec=0):
    import stkfmm_b200 as S
    fmm = S.StkWallFMM(p, max_pts, pbc, kernel, precision=prec)
    fmm.set_box(np.asarray(origin, dtype=np.float64), box)
    fmm.set_points(src, trg, None)
    fmm.setup_tree(kernel)
    out = np.zeros((len(trg), S.get_kernel_dimension(kernel)[2]))
    fmm.evaluate_fmm(kernel, val, out)
    return fmm, out


def rpy_values(rng, n, box=1.0):
    return np.concatenate([rng.normal(size=(n, 3)), rng.uniform(1e-4, 5e-4, (n, 1)) * box], axis=1)


@pytest.mark.parametrize("p", [8, 10])
def test_wall_stokes_matches_image_system(torch_cuda, p):
    rng = np.random.default_rng(50 + p)
    src = wall_points(rng, 4000)
    trg = np.concatenate([src[:1000], wall_points(rng, 1500)])
    f = rng.normal(size=(len(src), 3))
    _, out = run_wall(8, p, 50, 0, src, trg, f)
    ref = O.wall_stokes(src, f, trg)
    errs = component_errors(out, ref)
    assert max(errs) < TOL[p], errs


@pytest.mark.parametrize("p", [8, 10])
def test_wall_rpy_matches_image_system(torch_cuda, p):
    rng = np.random.default_rng(60 + p)
    src = wall_points(rng, 4000)
    trg = np.concatenate([src[:1000], wall_points(rng, 1500)])
    fb = rpy_values(rng, len(src))
    _, out = run_wall(16, p, 50, 0, src, trg, fb)
    ref = O.wall_rpy(src, fb, trg)
    errs = component_errors(out, ref)
    assert max(errs) < TOL[p], errs


@pytest.mark.parametrize("kernel", [8, 16])
@pytest.mark.parametrize("pbc", [0, 2])
def test_wall_no_slip(torch_cuda, kernel, pbc):
    """Targets on the wall get zero velocity (the reference's wall verification)."""
    rng = np.random.default_rng(70 + kernel + pbc)
    src = wall_points(rng, 3000)
    on_wall = rng.random((500, 3))
    on_wall[:, 2] = 0.0
    trg = np.concatenate([on_wall, src[:500]])
    val = rng.normal(size=(len(src), 3)) if kernel == 8 else rpy_values(rng, len(src))
    _, out = run_wall(kernel, 10, 50, pbc, src, trg, val)
    u_wall, u_bulk = out[:500, :3], out[500:, :3]
    assert np.linalg.norm(u_wall) / np.linalg.norm(u_bulk) < 1e-6


def test_wall_stokes_doubly_periodic(torch_cuda):
    """PXY: the image system over doubly periodic (Ewald) sums."""
    rng = np.random.default_rng(80)
    src = wall_points(rng, 600)
    trg = np.concatenate([src[:200], wall_points(rng, 200)])
    f = rng.normal(size=(len(src), 3))
    _, out = run_wall(8, 10, 32, 2, src, trg, f)
    ref = O.wall_stokes(src, f, trg, pbc=2)
    errs = component_errors(out, ref)
    assert max(errs) < TOL[10], errs


def test_wall_rpy_doubly_periodic_point_forces(torch_cuda):
    """PXY RPY with zero radii reduces to the Stokeslet wall system (its velocity)."""
    rng = np.random.default_rng(81)
    src = wall_points(rng, 600)
    trg = np.concatenate([src[:200], wall_points(rng, 200)])
    f = rng.normal(size=(len(src), 3))
    fb = np.concatenate([f, np.zeros((len(src), 1))], axis=1)
    _, out = run_wall(16, 10, 32, 2, src, trg, fb)
    ref = O.wall_stokes(src, f, trg, pbc=2)
    errs = component_errors(out[:, :3], ref)
    assert max(errs) < TOL[10], errs


@pytest.mark.parametrize("kernel", [8, 16])
def test_wall_box_scaling(torch_cuda, kernel):
    """A box (origin o, length L): the wall is z = o_z, results in physical units."""
    o, Lb = np.array([-1.0, 2.0, 0.5]), 3.0
    rng = np.random.default_rng(90 + kernel)
    src = wall_points(rng, 3000, box=Lb, origin=o)
    trg = np.concatenate([src[:500], wall_points(rng, 1000, box=Lb, origin=o)])
    val = rng.normal(size=(len(src), 3)) if kernel == 8 else rpy_values(rng, len(src), box=Lb)
    _, out = run_wall(kernel, 10, 50, 0, src, trg, val, box=Lb, origin=o)
    ref = O.wall_stokes(src, val, trg, z0=o[2]) if kernel == 8 else O.wall_rpy(src, val, trg, z0=o[2])
    errs = component_errors(out, ref)
    assert max(errs) < TOL[10], errs


@pytest.mark.parametrize("kernel", [8, 16])
def test_wall_mixed_and_device_entry(torch_cuda, kernel):
    """Mixed-precision P2P changes the wall result by ~1e-7; the device entry equals the host one."""
    torch = torch_cuda
    import stkfmm_b200 as S
    rng = np.random.default_rng(95 + kernel)
    src = wall_points(rng, 4000)
    trg = src.copy()
    val = rng.normal(size=(len(src), 3)) if kernel == 8 else rpy_values(rng, len(src))
    fmm, a = run_wall(kernel, 8, 50, 0, src, trg, val)
    _, b = run_wall(kernel, 8, 50, 0, src, trg, val, prec=S.PRECISION.MIXED)
    assert rel_l2(b, a) < 1e-6
    d_v = torch.as_tensor(val).cuda()
    d_o = torch.zeros(a.shape, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    fmm.evaluate_fmm_device(kernel, d_v.data_ptr(), d_o.data_ptr(), None)
    torch.cuda.synchronize()
    assert rel_l2(d_o.cpu().numpy(), a) < 1e-14
    assert fmm.last_kernel_ms() > 0


def test_wall_errors(torch_cuda):
    import stkfmm_b200 as S
    with pytest.raises(S.StkError):
        S.StkWallFMM(8, 50, S.PAXIS.PXYZ, 8)  # no wall image system for triply periodic boxes
    with pytest.raises(S.StkError):
        S.StkWallFMM(8, 50, 0, 1)  # neither Stokes nor RPY
    fmm = S.StkWallFMM(8, 50, 0, 8)
    fmm.set_box(np.zeros(3), 1.0)
    rng = np.random.default_rng(1)
    pts = wall_points(rng, 200)
    bad = pts.copy()
    bad[0, 2] = 0.6  # above the upper half of the box
    with pytest.raises(S.StkError):
        fmm.set_points(bad, pts, None)
    fmm.set_points(pts, pts, None)
    with pytest.raises(S.StkError):
        fmm.setup_tree(16)  # RPY not activated
    with pytest.raises(S.StkError):
        fmm.setup_tree(1)  # no wall system for LapPGrad
    with pytest.raises(S.StkError):
        fmm.evaluate_fmm(8, np.zeros((200, 3)), np.zeros((200, 3)))  # before setup_tree
