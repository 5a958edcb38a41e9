"""GPU: triply periodic (PXYZ) evaluate_fmm against the oracle's Ewald sums.

The oracle (oracle/stk_oracle.c:oracle_ewald) restates the periodic Green's
functions of the reference's M2C generator (M2L/Laplace/Laplace3D3D.cpp,
M2L/Stokeslet/Stokes3D3D.cpp) and is itself checked for independence of the
Ewald split and against lattice sums (tests/test_oracle.py); the reference's
extra PXYZ terms (PVel net flux and net force, the Laplace neutraliser) are
oracle.pvel_pxyz_terms and oracle.laplace_pxyz_neutraliser.  Inputs follow the
reference's periodic tests: net force (charge) removed (Test/Test.cpp:332-351),
except where a test says otherwise.  Error measure: relative L2 per output
component (Test/Test.cpp:113-151).
"""
import numpy as np
import pytest

from conftest import component_errors
from helpers import clustered_points
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = {8: 2e-5, 10: 2e-6}


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def points(kind, n, seed):
    rng = np.random.default_rng(seed)
    if kind == "uniform":
        return rng.random((n, 3)), rng
    return np.minimum(clustered_points(rng, n, nclusters=5, sigma=0.05), 0.999), rng


def periodic_fmm(kernel, p, max_pts, pts, slv):
    import stkfmm_b200 as S
    fmm = S.Stk3DFMM(p, max_pts, S.PAXIS.PXYZ, kernel)
    fmm.set_box(np.zeros(3), 1.0)
    fmm.set_points(pts, pts, None)
    fmm.setup_tree(kernel)
    out = np.zeros((len(pts), S.get_kernel_dimension(kernel)[2]))
    fmm.evaluate_fmm(kernel, slv, out, None)
    return fmm, out


@pytest.mark.parametrize("dist", ["uniform", "clustered"])
@pytest.mark.parametrize("p", [8, 10])
def test_periodic_stokes(torch_cuda, dist, p):
    pts, rng = points(dist, 5000, 3)
    f = rng.normal(size=(len(pts), 3))
    f -= f.mean(0)
    fmm, out = periodic_fmm(8, p, 64, pts, f)
    ref = O.ewald(O.EWALD_STOKES, pts, f, pts)
    errs = component_errors(out, ref)
    assert max(errs) < TOL[p], errs


@pytest.mark.parametrize("p", [8, 10])
def test_periodic_laplace(torch_cuda, p):
    pts, rng = points("clustered", 5000, 4)
    q = rng.uniform(-0.5, 0.5, (len(pts), 1))
    q -= q.mean()
    _, out = periodic_fmm(1, p, 64, pts, q)
    ref = O.ewald(O.EWALD_LAPLACE, pts, q, pts)
    # the periodic potential is defined up to a constant: compare it with the mean removed
    out[:, 0] -= out[:, 0].mean()
    ref[:, 0] -= ref[:, 0].mean()
    errs = component_errors(out, ref)
    assert max(errs) < TOL[p], errs


def test_periodic_rpy_velocity(torch_cuda):
    """RPY (u, lap u): u against Ewald Stokeslet + the finite-radius terms of the
    27 nearest images (beyond those, b^2/r^3 terms are below 1e-8)."""
    pts, rng = points("uniform", 4000, 5)
    f = rng.normal(size=(len(pts), 3))
    f -= f.mean(0)
    b = rng.uniform(1e-4, 5e-4, len(pts))
    slv = np.concatenate([f, b[:, None]], axis=1)
    _, out = periodic_fmm(16, 10, 64, pts, slv)
    ref = O.ewald(O.EWALD_STOKES, pts, f, pts)
    r = np.arange(-1, 2)
    shifts = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3).astype(np.float64)
    imgs = (pts[None] + shifts[:, None]).reshape(-1, 3)
    corr = O.direct(O.UK_RPY_U, imgs, np.tile(slv, (27, 1)), pts) - O.direct(O.UK_STOKES_VEL, imgs,
                                                                            np.tile(f, (27, 1)), pts)
    errs = component_errors(out[:, :3], ref + corr)
    assert max(errs) < TOL[10], errs


def test_periodic_rpy_laplacian(torch_cuda):
    """RPY's lap u (no radius term) against the periodic Laplacian of the
    Stokeslet sum (oracle.ewald_stokes_laplacian, pinned by finite differences in
    tests/test_oracle.py).  The images beyond the cell carry 1.3-1.9% of it on
    these points, so a bar of 1e-4 catches any error above ~1% of theirs."""
    pts, rng = points("uniform", 4000, 5)
    f = rng.normal(size=(len(pts), 3))
    f -= f.mean(0)
    b = rng.uniform(1e-4, 5e-4, len(pts))
    _, out = periodic_fmm(16, 10, 64, pts, np.concatenate([f, b[:, None]], axis=1))
    errs = component_errors(out[:, 3:6], O.ewald_stokes_laplacian(pts, f, pts))
    assert max(errs) < 1e-4, errs


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_rpy_pxyz_2m_against_ewald(torch_cuda, precision):
    """The full-size RPY PXYZ workload (2,097,152 uniform points, p = 8, 256 points per
    leaf) against its Ewald-summed fixture at 4,096 sampled targets (u and lap u,
    tests/golden/make_rpy_pxyz_ewald.py).  Bars: the per-component relative L2 errors
    measured on B200 (FP64 and mixed), with headroom of about 2x."""
    import os
    import sys
    import stkfmm_b200 as S
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    sys.path.insert(0, here)
    import make_rpy_pxyz_ewald as G
    z = np.load(os.path.join(here, "rpy_pxyz_2m_ewald.npz"))
    pts, f, b = G.workload()
    assert (z["idx"] == G.sample()).all()
    slv = np.concatenate([f, b], axis=1)
    fmm = S.Stk3DFMM(8, 256, S.PAXIS.PXYZ, 16)
    fmm.set_box(np.zeros(3), 1.0)
    fmm.set_points(pts, pts, None)
    fmm.setup_tree(16)
    fmm.set_precision(S.PRECISION.FP64 if precision == "fp64" else S.PRECISION.MIXED)
    out = np.zeros((len(pts), 6))
    fmm.evaluate_fmm(16, slv, out, None)
    errs = component_errors(out[z["idx"]], z["truth"])
    print(precision, errs)
    assert max(errs[:3]) < RPY2M_TOL[precision][0], errs
    assert max(errs[3:]) < RPY2M_TOL[precision][1], errs


# (u, lap u) bars of test_rpy_pxyz_2m_against_ewald
RPY2M_TOL = {"fp64": (1e-3, 1e-3), "mixed": (1e-3, 1e-3)}


def test_periodic_mixed_close_to_fp64(torch_cuda):
    import stkfmm_b200 as S
    pts, rng = points("clustered", 5000, 6)
    f = rng.normal(size=(len(pts), 3))
    f -= f.mean(0)
    res = []
    for prec in (S.PRECISION.FP64, S.PRECISION.MIXED):
        fmm = S.Stk3DFMM(10, 64, S.PAXIS.PXYZ, 8, precision=prec)
        fmm.set_box(np.zeros(3), 1.0)
        fmm.set_points(pts, pts, None)
        fmm.setup_tree(8)
        out = np.zeros((len(pts), 3))
        fmm.evaluate_fmm(8, f, out, None)
        res.append(out)
    assert np.linalg.norm(res[1] - res[0]) / np.linalg.norm(res[0]) < 1e-6


def periodic_fmm_pbc(kernel, pbc, p, max_pts, pts, slv):
    import stkfmm_b200 as S
    fmm = S.Stk3DFMM(p, max_pts, pbc, kernel)
    fmm.set_box(np.zeros(3), 1.0)
    fmm.set_points(pts, pts, None)
    fmm.setup_tree(kernel)
    out = np.zeros((len(pts), S.get_kernel_dimension(kernel)[2]))
    fmm.evaluate_fmm(kernel, slv, out, None)
    return out


@pytest.mark.parametrize("dist", ["uniform", "clustered"])
def test_doubly_periodic_stokes(torch_cuda, dist):
    pts, rng = points(dist, 2000, 7)
    f = rng.normal(size=(len(pts), 3))
    f -= f.mean(0)
    out = periodic_fmm_pbc(8, 2, 10, 50, pts, f)
    ref = O.ewald2d(O.EWALD_STOKES, pts, f, pts)
    errs = component_errors(out, ref)
    assert max(errs) < TOL[10], errs


def test_doubly_periodic_laplace(torch_cuda):
    pts, rng = points("clustered", 2000, 8)
    q = rng.uniform(-0.5, 0.5, (len(pts), 1))
    q -= q.mean()
    out = periodic_fmm_pbc(1, 2, 10, 50, pts, q)
    ref = O.ewald2d(O.EWALD_LAPLACE, pts, q, pts)
    out[:, 0] -= out[:, 0].mean()
    ref[:, 0] -= ref[:, 0].mean()
    errs = component_errors(out, ref)
    assert max(errs) < TOL[10], errs


@pytest.mark.parametrize("pbc", [2, 3])
def test_periodic_pvel(torch_cuda, pbc):
    """StokesPVel (pressure and velocity) with f and trD, neutralised as the
    reference's periodic tests do (Test/Test.cpp:364-402).  PXYZ follows the
    reference's conventions (oracle.pvel_pxyz_terms: half the trD dipole moment
    on the velocity), which leave the velocity without drift; the triply periodic
    pressure is fixed only up to a constant, the "drift" the reference's error
    measure reports apart from the error (mean difference per component,
    Test/Test.cpp:143-150), and is compared with it removed.  PXY has none."""
    pts, rng = points("clustered", 2000, 9 + pbc)
    v = rng.normal(size=(len(pts), 4))
    v -= v.mean(0)
    out = periodic_fmm_pbc(128, pbc, 10, 50, pts, v)
    if pbc == 2:
        ref = O.ewald2d(O.EWALD_PVEL, pts, v, pts)
    else:
        ref = O.ewald(O.EWALD_PVEL, pts, v, pts) + O.pvel_pxyz_terms(pts, v, pts)
        out[:, 0] -= (out[:, 0] - ref[:, 0]).mean()
    errs = component_errors(out, ref)
    assert max(errs) < TOL[10], errs


def test_periodic_pvel_family_net_flux(torch_cuda):
    """PXYZ PVelGrad and PVelLaplacian share PVel's far field and its net-flux
    correction (FMMData.cpp:214-216 names all three): their pressure and velocity
    equal PVel's; and the velocity carries half the trD dipole moment, which a
    shift of the trD sources changes (the reference's M2C is not translation
    invariant, StokesPVel3D3D.cpp:362-364)."""
    pts, rng = points("uniform", 2000, 31)
    v = np.zeros((len(pts), 4))
    v[:, 3] = rng.normal(size=len(pts))
    v[:, 3] -= v[:, 3].mean()
    res = {}
    for k in (128, 256, 512):
        res[k] = periodic_fmm_pbc(k, 3, 10, 50, pts, v)
    for k in (256, 512):
        assert np.linalg.norm(res[k][:, :4] - res[128]) / np.linalg.norm(res[128]) < 1e-11, k
    ref = O.ewald(O.EWALD_PVEL, pts, v, pts) + O.pvel_pxyz_terms(pts, v, pts)
    errs = component_errors(res[128][:, 1:], ref[:, 1:])
    assert max(errs) < TOL[10], errs


def test_periodic_laplace_charged(torch_cuda):
    """A charged cell: the reference's PXYZ Laplace operator pairs every
    equivalent charge with an opposite one at the cell centre
    (M2L/Laplace/Laplace3D3D.cpp:266-273; oracle.laplace_pxyz_neutraliser).
    The gradient is compared as is, the potential with its drift removed."""
    pts, rng = points("clustered", 2000, 33)
    q = rng.normal(size=(len(pts), 1)) + 0.2
    out = periodic_fmm_pbc(1, 3, 10, 50, pts, q)
    ref = O.ewald(O.EWALD_LAPLACE, pts, q, pts) + O.laplace_pxyz_neutraliser(q.sum(), pts)
    out[:, 0] -= (out[:, 0] - ref[:, 0]).mean()
    errs = component_errors(out, ref)
    assert max(errs) < TOL[10], errs


def test_periodic_translation(torch_cuda):
    """Shifting every point by a vector (wrapped into the cell) gives the same
    values, up to the per-component drift (the reference's translation check,
    Test/Test.cpp:646-673)."""
    pts, rng = points("uniform", 3000, 12)
    f = rng.normal(size=(len(pts), 3))
    f -= f.mean(0)
    a = periodic_fmm_pbc(8, 3, 10, 50, pts, f)
    b = periodic_fmm_pbc(8, 3, 10, 50, np.mod(pts + np.array([0.31, 0.17, 0.73]), 1.0), f)
    d = (b - a).mean(0)
    assert max(component_errors(b - d, a)) < TOL[10]


@pytest.mark.parametrize("kernel,pbc", [(8, 3), (1, 2), (128, 1)])
def test_far_field_off_sums_two_cells(torch_cuda, kernel, pbc):
    """Far field off (the reference's enableFF = false, FMMData.cpp:83-89): no
    far-image operator, so the periodic sum stops at the images within two cells
    on each periodic axis, the images PVFMM's periodic lists reach (the block its
    M2C generators leave to the tree, DIRECTLAYER = 2).  Compared with that finite
    lattice sum, summed directly by the oracle; the values need no neutrality."""
    import stkfmm_b200 as S
    pts, rng = points("clustered", 1500, 70 + pbc)
    v = rng.normal(size=(len(pts), S.get_kernel_dimension(kernel)[0]))
    fmm = S.Stk3DFMM(10, 50, pbc, kernel, enable_ff=False)
    fmm.set_box(np.zeros(3), 1.0)
    fmm.set_points(pts, pts, None)
    fmm.setup_tree(kernel)
    out = np.zeros((len(pts), S.get_kernel_dimension(kernel)[2]))
    fmm.evaluate_fmm(kernel, v, out, None)
    r = range(-2, 3)
    shifts = np.array([(a, b, c) for a in r for b in (r if pbc >= 2 else [0]) for c in (r if pbc == 3 else [0])],
                      dtype=np.float64)
    imgs = (pts[None] + shifts[:, None]).reshape(-1, 3)
    ref = O.direct(S.kernel_slot(kernel, 0), imgs, np.tile(v, (len(shifts), 1)), pts)
    errs = component_errors(out, ref)
    assert max(errs) < TOL[10], errs
    # switching it back on needs a new setup_tree, then gives the full periodic sum
    fmm.set_far_field(True)
    with pytest.raises(S.StkError):
        fmm.evaluate_fmm(kernel, v, out, None)


@pytest.mark.parametrize("kernel", [1, 2, 4, 8, 128, 256, 1024])
def test_singly_periodic_against_image_sum(torch_cuda, kernel):
    """PX: sources without net charge / force, dipole or quadrupole (alternating
    signs on the corners of small cubes) against the direct sum over their
    images |t| <= 3000 along x (the tail beyond is far below the bar)."""
    import itertools
    import stkfmm_b200 as S
    rng = np.random.default_rng(40 + kernel)
    c = rng.random((16, 3)) * 0.8 + 0.1
    sg = np.array(list(itertools.product([-1, 1], [-1, 1], [-1, 1])), dtype=np.float64)
    src = np.concatenate([ci + 0.03 * sg for ci in c])
    s = np.tile(sg.prod(1), 16)[:, None]
    quad = s * np.array([[0.4, 0.1, -0.3, 0.2, -0.5, 0.3, 0.1, 0.6, 0.2]])
    fv = np.concatenate([s * np.array([[0.3, -0.2, 0.5]]), 0.7 * s], axis=1)
    val = {1: s, 2: s, 4: quad, 8: s * np.array([[0.3, -0.2, 0.5]]), 256: fv, 1024: fv,
           128: np.concatenate([s * np.array([[0.3, -0.2, 0.5]]), 0.7 * s], axis=1)}[kernel]
    trg = rng.random((1500, 3)) * 0.999
    fmm = S.Stk3DFMM(10, 32, S.PAXIS.PX, kernel)
    fmm.set_box(np.zeros(3), 1.0)
    fmm.set_points(src, trg, None)
    fmm.setup_tree(kernel)
    out = np.zeros((len(trg), S.get_kernel_dimension(kernel)[2]))
    fmm.evaluate_fmm(kernel, val, out, None)
    T = 3000
    sh = np.zeros((2 * T + 1, 3))
    sh[:, 0] = np.arange(-T, T + 1)
    imgs = (src[None] + sh[:, None]).reshape(-1, 3)
    uk = S.kernel_slot(kernel, 0)
    ref = O.direct(uk, imgs, np.tile(val, (len(sh), 1)), trg)
    errs = component_errors(out, ref)
    assert max(errs) < TOL[10], errs


@pytest.mark.parametrize("pbc", [2, 3])
def test_periodic_laplace_hessian(torch_cuda, pbc):
    """LapPGradGrad (potential, gradient, Hessian) against the oracle's Ewald
    sums with the Hessian (PXYZ potential compared with the mean removed)."""
    pts, rng = points("clustered", 3000, 13 + pbc)
    q = rng.uniform(-0.5, 0.5, (len(pts), 1))
    q -= q.mean()
    out = periodic_fmm_pbc(2, pbc, 10, 50, pts, q)
    ref = (O.ewald if pbc == 3 else O.ewald2d)(O.EWALD_LAPLACE_HESS, pts, q, pts)
    if pbc == 3:
        out[:, 0] -= out[:, 0].mean()
        ref[:, 0] -= ref[:, 0].mean()
    errs = component_errors(out, ref)
    assert max(errs) < TOL[10], errs


@pytest.mark.parametrize("pbc", [2, 3])
def test_periodic_quadrupole_potential(torch_cuda, pbc):
    """LapQPGradGrad's potential S : grad grad G summed over the periodic images,
    from the oracle's Ewald Hessians (one sum per symmetric component of S; the
    PXYZ potential compared with the mean removed)."""
    pts, rng = points("clustered", 2000, 15 + pbc)
    S = rng.uniform(-1, 1, (len(pts), 9))
    out = periodic_fmm_pbc(4, pbc, 10, 50, pts, S)
    ew = O.ewald if pbc == 3 else O.ewald2d
    ref = np.zeros(len(pts))
    for col, (i, j) in enumerate(((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))):
        w = S[:, 3 * i + j] + (S[:, 3 * j + i] if i != j else 0.0)
        ref += ew(O.EWALD_LAPLACE_HESS, pts, w[:, None], pts)[:, 4 + col]
    pot = out[:, 0].copy()
    if pbc == 3:
        pot -= pot.mean()
        ref -= ref.mean()
    assert np.linalg.norm(pot - ref) / np.linalg.norm(ref) < TOL[10]


@pytest.mark.parametrize("kernel,pbc", [(8, 3), (1, 2)])
def test_complete_level_m2l_matches_chunked(torch_cuda, monkeypatch, kernel, pbc):
    """The per-type M2L of complete levels (4096 boxes at level 4 here) gives the
    chunked per-offset M2L's result; STKFMM_M2L_DENSE=0 selects the chunked one."""
    import stkfmm_b200 as S
    pts, rng = points("uniform", 20000, 30 + kernel)
    v = rng.normal(size=(len(pts), S.get_kernel_dimension(kernel)[0]))
    v -= v.mean(0)
    res = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("STKFMM_M2L_DENSE", mode)
        fmm = S.Stk3DFMM(6, 8, pbc, kernel)
        fmm.set_box(np.zeros(3), 1.0)
        fmm.set_points(pts, pts, None)
        fmm.setup_tree(kernel)
        out = np.zeros((len(pts), S.get_kernel_dimension(kernel)[2]))
        fmm.evaluate_fmm(kernel, v, out, None)
        res[mode] = (out, fmm.m2l_work(kernel), fmm.tree_stats(kernel))
    assert res["1"][2]["depth"] >= 4
    # the dense path ran: no padded ranks or columns executed
    assert res["1"][1]["flops_executed"] < res["0"][1]["flops_executed"]
    assert res["1"][1]["flops_algorithmic"] == res["0"][1]["flops_algorithmic"]
    a, b = res["0"][0], res["1"][0]
    assert np.linalg.norm(b - a) / np.linalg.norm(a) < 1e-13


@pytest.mark.parametrize("pbc", [0, 2, 3])
def test_traction_is_stress_of_pvelgrad(torch_cuda, pbc):
    """The Traction FMM equals -p I + grad u + grad u^T of the PVelGrad FMM on the
    same points and SL + DL values (both share the stokes_PVel far field; the
    identity holds pair by pair for the reference's kernels, tests/test_oracle.py),
    free space and periodic."""
    import stkfmm_b200 as S
    pts, rng = points("clustered", 3000, 60 + pbc)
    v = rng.normal(size=(len(pts), 4))
    v -= v.mean(0)
    d = rng.normal(size=(len(pts), 9))
    d[:, [0, 4, 8]] -= (d[:, 0] + d[:, 4] + d[:, 8]).mean() / 3
    res = {}
    for k in (256, 1024):
        fmm = S.Stk3DFMM(8, 50, pbc, k)
        fmm.set_box(np.zeros(3), 1.0)
        fmm.set_points(pts, pts, pts)
        fmm.setup_tree(k)
        out = np.zeros((len(pts), S.get_kernel_dimension(k)[2]))
        fmm.evaluate_fmm(k, v, out, d)
        res[k] = out
    g = res[256][:, 7:16].reshape(-1, 3, 3)
    comb = (-res[256][:, 0][:, None, None] * np.eye(3)[None] + g + g.transpose(0, 2, 1)).reshape(-1, 9)
    assert np.linalg.norm(comb - res[1024]) / np.linalg.norm(res[1024]) < 1e-10
