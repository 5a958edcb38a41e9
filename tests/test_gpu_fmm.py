"""GPU: Stk3DFMM_evaluate_fmm (U-list near field + KIFMM far field) against the
direct sum of the oracle, with the reference's error measure (relative L2 per
output component, Test/Test.cpp:113-151).

The KIFMM truncation error falls with the multipole order p; the bars below
are per-component relative L2 errors of the FP64 path at that order on
clustered (adaptive-tree) inputs, the cases the reference's own tests run
(Test/main.cpp: p = 8 .. 16, max_pts = 50 .. 2000).
"""
import numpy as np
import pytest

from conftest import component_errors, rel_l2
from helpers import clustered_points, uk_values
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# per-component relative L2 bar at multipole order p (FP64 path)
FMM_TOL = {6: 2e-4, 8: 2e-5, 10: 2e-6, 12: 2e-7}


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def fmm_case(kernel, n, seed, box=1.0, origin=(0.0, 0.0, 0.0)):
    import stkfmm_b200 as S
    rng = np.random.default_rng(seed)
    pts = np.minimum(clustered_points(rng, n, nclusters=5, sigma=0.05), 0.999) * box + np.array(origin)
    sd, dd, td = S.get_kernel_dimension(kernel)
    has_dl = S.kernel_slot(kernel, 1) >= 0
    slv = uk_values(rng, S.kernel_slot(kernel, 0), n)
    if kernel in (16, 32):
        # RPY radii / regularization lengths well below the leaf sizes: S2M and S2L
        # use the regularized / finite-size kernel while M2T, L2T and the
        # translations use the plain Stokeslet (the reference's kernel
        # compositions), a model difference of relative size (eps / r)^2
        slv[:, 3] = rng.uniform(1e-4, 5e-4, n) * box
    if kernel == 64:
        slv[:, 6] = rng.uniform(1e-4, 5e-4, n) * box  # regularisation, as above
    dlv = rng.normal(size=(n, dd)) if has_dl else None
    return pts, slv, dlv, td


def direct_truth(kernel, pts, slv, dlv):
    """The whole sum with the kernel's S2T micro-kernels (SL and DL), in the unit box."""
    import stkfmm_b200 as S
    ref = O.direct(S.kernel_slot(kernel, 0), pts, slv, pts)
    if dlv is not None:
        ref += O.direct(S.kernel_slot(kernel, 1), pts, dlv, pts)
    return ref


def run_fmm(kernel, p, max_pts, pts, slv, dlv, td, prec=0, box=1.0, origin=(0.0, 0.0, 0.0)):
    import stkfmm_b200 as S
    fmm = S.Stk3DFMM(p, max_pts, 0, kernel, precision=prec)
    fmm.set_box(np.asarray(origin, dtype=np.float64), box)
    fmm.set_points(pts, pts, pts if dlv is not None else None)
    fmm.setup_tree(kernel)
    out = np.zeros((len(pts), td))
    fmm.evaluate_fmm(kernel, slv, out, dlv)
    return fmm, out


@pytest.mark.parametrize("kernel", [1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024])
@pytest.mark.parametrize("p", [6, 8, 10])
def test_fmm_matches_direct_sum(torch_cuda, kernel, p):
    pts, slv, dlv, td = fmm_case(kernel, 6000, seed=10 + kernel)
    fmm, out = run_fmm(kernel, p, 50, pts, slv, dlv, td)
    ref = direct_truth(kernel, pts, slv, dlv)
    errs = component_errors(out, ref)
    st = fmm.tree_stats(kernel)
    # an adaptive tree: every far-field list is exercised
    assert st["v_entries"] > 0 and st["w_entries"] > 0 and st["x_entries"] > 0, st
    assert max(errs) < FMM_TOL[p], (p, errs)


@pytest.mark.parametrize("kernel", [1, 8])
def test_fmm_higher_order(torch_cuda, kernel):
    pts, slv, dlv, td = fmm_case(kernel, 8000, seed=3)
    _, out = run_fmm(kernel, 12, 100, pts, slv, dlv, td)
    errs = component_errors(out, direct_truth(kernel, pts, slv, dlv))
    assert max(errs) < FMM_TOL[12], errs


@pytest.mark.parametrize("kernel", [1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024])
def test_fmm_mixed_close_to_fp64(torch_cuda, kernel):
    """The mixed-precision P2P passes change the FMM result by ~1e-7 at most."""
    pts, slv, dlv, td = fmm_case(kernel, 6000, seed=20 + kernel)
    _, a = run_fmm(kernel, 8, 50, pts, slv, dlv, td, prec=0)
    _, b = run_fmm(kernel, 8, 50, pts, slv, dlv, td, prec=1)
    assert rel_l2(b, a) < 1e-6


def test_fmm_repeatable_and_device_entry(torch_cuda):
    """Two evaluations in a row agree bit for bit; the device entry point matches the host one."""
    torch = torch_cuda
    kernel = 1
    pts, slv, dlv, td = fmm_case(kernel, 5000, seed=7)
    fmm, a = run_fmm(kernel, 8, 64, pts, slv, dlv, td)
    b = np.zeros_like(a)
    fmm.evaluate_fmm(kernel, slv, b, dlv)
    assert np.array_equal(a, b)
    d_sl = torch.as_tensor(slv).cuda()
    d_dl = torch.as_tensor(dlv).cuda()
    d_out = torch.zeros((len(pts), td), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    fmm.evaluate_fmm_device(kernel, d_sl.data_ptr(), d_out.data_ptr(), d_dl.data_ptr(), None)
    torch.cuda.synchronize()
    assert rel_l2(d_out.cpu().numpy(), a) < 1e-14


@pytest.mark.parametrize("kernel", [1, 2, 4, 16, 128])
def test_fmm_box_scaling(torch_cuda, kernel):
    """A box (origin o, length L): FMM in physical units equals the direct sum in physical units."""
    import stkfmm_b200 as S
    o, Lb = np.array([-1.0, 2.0, 0.5]), 3.0
    pts, slv, dlv, td = fmm_case(kernel, 5000, seed=30 + kernel, box=Lb, origin=o)
    _, out = run_fmm(kernel, 10, 64, pts, slv, dlv, td, box=Lb, origin=o)
    ref = direct_truth(kernel, pts, slv, dlv)
    errs = component_errors(out, ref)
    assert max(errs) < FMM_TOL[10], errs


def test_fmm_separate_targets(torch_cuda):
    """Targets apart from the sources (a uniform cloud), Stokes."""
    import stkfmm_b200 as S
    rng = np.random.default_rng(11)
    src = np.minimum(clustered_points(rng, 4000, nclusters=4, sigma=0.05), 0.999)
    trg = rng.random((3000, 3)) * 0.999
    f = rng.normal(size=(len(src), 3))
    fmm = S.Stk3DFMM(10, 50, 0, 8)
    fmm.set_box(np.zeros(3), 1.0)
    fmm.set_points(src, trg, None)
    fmm.setup_tree(8)
    out = np.zeros((len(trg), 3))
    fmm.evaluate_fmm(8, f, out, None)
    ref = O.direct(S.kernel_slot(8, 0), src, f, trg)
    assert max(component_errors(out, ref)) < FMM_TOL[10]


def test_fmm_not_supported_cases(torch_cuda):
    import stkfmm_b200 as S
    pts = np.random.default_rng(0).random((500, 3))
    with pytest.raises(S.StkError):
        S.Stk3DFMM(8, 50, 0, 2048)  # no STKFMM kernel has this bit
    lg = S.Stk3DFMM(8, 50, 0, 1)
    lg.set_box(np.zeros(3), 1.0)
    lg.set_points(pts, pts, pts)
    with pytest.raises(S.StkError):
        lg.setup_tree(64)  # not activated in this handle


@pytest.mark.parametrize("pbc", [0, 3])
def test_operators_shared_between_handles(torch_cuda, pbc):
    """A second handle of the same (translation kernel, p) reuses the first handle's
    far-field operators (and periodic M2C): its first evaluation does no operator
    build, and both handles give the same answer as a handle that built its own."""
    import time
    import stkfmm_b200 as S
    rng = np.random.default_rng(77 + pbc)
    n = 6000
    pts = rng.random((n, 3))
    q = rng.uniform(-0.5, 0.5, (n, 1))
    q -= q.mean()  # a neutral cell for the periodic sum

    def first_eval(fmm):
        out = np.zeros((n, 4))
        t0 = time.perf_counter()
        fmm.evaluate_fmm(1, q, out, None)
        return time.perf_counter() - t0, out

    def handle():
        f = S.Stk3DFMM(10, 128, pbc, 1)
        f.set_box(np.zeros(3), 1.0)
        f.set_points(pts, pts, None)
        f.setup_tree(1)
        return f

    a = handle()
    ta, oa = first_eval(a)
    b = handle()  # a is alive: b aliases its operators
    tb, ob = first_eval(b)
    assert tb < 0.5 * ta, (ta, tb)
    assert rel_l2(ob, oa) < 1e-13
    del a, b
    c = handle()  # no holder left: c builds its own
    tc, oc = first_eval(c)
    assert rel_l2(oc, oa) < 1e-13


@pytest.mark.parametrize("kernel,p", [(1, 10), (8, 8), (128, 8)])
def test_mixed_chunked_m2l_tensor_cores(torch_cuda, monkeypatch, kernel, p):
    """The mixed path's per-offset (chunked) M2L on the tensor cores (grouped 3xTF32
    tcgen05 GEMMs) is as accurate as the same M2L in SIMT FP32 (STKFMM_M2L_TC=0): the
    mixed FMM stays within 1e-6 of FP64, on an adaptive clustered tree whose levels
    all take the chunked path."""
    import stkfmm_b200 as S
    pts, slv, dlv, td = fmm_case(kernel, 12000, seed=40 + kernel)
    res = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("STKFMM_M2L_TC", mode)
        _, res[mode] = run_fmm(kernel, p, 40, pts, slv, dlv, td, prec=1)
    _, ref = run_fmm(kernel, p, 40, pts, slv, dlv, td, prec=0)
    # both FP32-accurate: each within 1e-6 of FP64, the tensor-core one no worse
    e1, e0 = rel_l2(res["1"], ref), rel_l2(res["0"], ref)
    assert e1 < 1e-6 and e1 < 1.5 * e0 + 1e-7, (e1, e0)
    # relative to the part beyond the U-list near field (what the far field computes, plus
    # the direct W / X pairs), the tensor-core M2L's mixed FMM errs no more than the SIMT one's
    fmm = S.Stk3DFMM(p, 40, 0, kernel)
    fmm.set_box(np.zeros(3), 1.0)
    fmm.set_points(pts, pts, pts if dlv is not None else None)
    fmm.setup_tree(kernel)
    near = np.zeros_like(ref)
    fmm.evaluate_near(kernel, slv, near, dlv)
    far = ref - near
    e_tc, e_simt = rel_l2(res["1"] - ref, far), rel_l2(res["0"] - ref, far)
    assert e_tc < 1.5 * e_simt + 1e-7, (e_tc, e_simt)
