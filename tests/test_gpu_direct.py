"""GPU parity: dense direct sums (STKFMM::evaluateKernel path) through the C ABI.

FP64 must match the oracle to 1e-12 relative L2; the mixed path to 1e-6.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2
from helpers import UK_FORWARD, GOLDEN_MAP, UK_NAMES, UK_SDIM, UK_TDIM, load_golden, uk_values
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = {0: 1e-12, 1: 1e-6}


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


@pytest.fixture(scope="module")
def L():
    from stkfmm_b200 import lib
    return lib()


def dev(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def gpu_direct(torch, L, uk, src, val, trg, prec, out0=None):
    td = UK_TDIM[uk]
    s, v, t = dev(torch, src), dev(torch, val), dev(torch, trg)
    o = dev(torch, out0) if out0 is not None else torch.zeros((len(trg), td), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.stk_ukernel_direct_device(uk, len(src), s.data_ptr(), v.data_ptr(), len(trg), t.data_ptr(),
                                     o.data_ptr(), prec, stream)
    assert rc == 0, rc
    torch.cuda.synchronize()
    return o.cpu().numpy()


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("name", sorted(GOLDEN_MAP))
def test_direct_golden(torch_cuda, L, name, prec):
    """Reference SimpleKernel fixtures reproduced on the GPU (random and fixed-point layouts)."""
    g = load_golden(name)
    for uk, osl, vsl in GOLDEN_MAP[name]:
        for pre in ("", "fixed_"):
            out = gpu_direct(torch_cuda, L, uk, g[pre + "src"], g[pre + "val"][:, vsl], g[pre + "trg"], prec)
            err = rel_l2(out, g[pre + "out"][:, osl])
            assert err < TOL[prec], (name, UK_NAMES[uk], pre, prec, err)


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("uk", UK_FORWARD)
def test_direct_all_ukernels_vs_oracle(torch_cuda, L, uk, prec):
    rng = np.random.default_rng(100 + uk)
    src = rng.random((3000, 3))
    trg = np.concatenate([src[:500], rng.random((700, 3))])
    val = uk_values(rng, uk, len(src))
    out = gpu_direct(torch_cuda, L, uk, src, val, trg, prec)
    if uk == 11:  # fused laplace SL+DL
        ref = O.direct(1, src, val[:, :1], trg) + O.direct(3, src, val[:, 1:4], trg)
    elif uk == 12:  # fused stokes SL+DL
        ref = O.direct(9, src, val[:, :4], trg) + O.direct(10, src, val[:, 4:13], trg)
    elif uk == 15:  # fused laplace SL+DL potential
        ref = O.direct(0, src, val[:, :1], trg) + O.direct(2, src, val[:, 1:4], trg)
    else:
        ref = O.direct(uk, src, val, trg)
    assert rel_l2(out, ref) < TOL[prec], (UK_NAMES[uk], rel_l2(out, ref))


@pytest.mark.parametrize("ns,nt", [(0, 10), (10, 0), (1, 1), (5, 1), (37, 33), (1000, 31), (257, 1025)])
def test_direct_ragged_and_empty(torch_cuda, L, ns, nt):
    rng = np.random.default_rng(ns * 1000 + nt)
    src = rng.random((ns, 3))
    trg = rng.random((nt, 3))
    val = uk_values(rng, 6, ns)
    out0 = rng.normal(size=(nt, 6))
    if ns == 0 or nt == 0:
        s = np.zeros((max(ns, 1), 3))
        out = out0.copy()
        rc = L.stk_ukernel_direct_device(6, ns, 0, 0, nt, 0, 0, 0, 0)
        assert rc == 0
        return
    out = gpu_direct(torch_cuda, L, 6, src, val, trg, 0, out0=out0)
    ref = O.direct(6, src, val, trg, out=out0.copy())
    assert rel_l2(out, ref) < 1e-12


def test_direct_large_split_sources(torch_cuda, L):
    """Few targets, many sources: the source range is split across items with atomic accumulation."""
    rng = np.random.default_rng(5)
    src = rng.random((60000, 3))
    trg = rng.random((64, 3))
    val = uk_values(rng, 4, len(src))
    out = gpu_direct(torch_cuda, L, 4, src, val, trg, 0)
    ref = O.direct(4, src, val, trg)
    assert rel_l2(out, ref) < 1e-12
    out = gpu_direct(torch_cuda, L, 4, src, val, trg, 1)
    assert rel_l2(out, ref) < 1e-6


KERNELS = {1: (1, 3, 4), 2: (1, 3, 10), 4: (9, None, 10), 8: (3, None, 3), 16: (4, None, 6), 32: (4, None, 3),
           64: (7, None, 6), 128: (4, 9, 4), 256: (4, 9, 16), 512: (4, 9, 7), 1024: (4, 9, 9)}


@pytest.mark.parametrize("kernel", sorted(KERNELS))
@pytest.mark.parametrize("prec", [0, 1])
def test_evaluate_kernel_host_api(torch_cuda, kernel, prec):
    """stk_evaluate_kernel (host arrays, accumulate) for SLS2T, DLS2T and L2T."""
    import stkfmm_b200 as S
    rng = np.random.default_rng(kernel)
    src = rng.random((900, 3)) * 3.0 - 1.0  # raw coordinates, no box scaling
    trg = np.concatenate([src[:100], rng.random((300, 3))])
    sd, dd, td = S.get_kernel_dimension(kernel)
    for p2p, slot in ((S.PPKERNEL.SLS2T, 0), (S.PPKERNEL.DLS2T, 1), (S.PPKERNEL.L2T, 6)):
        uk = S.kernel_slot(kernel, slot)
        out0 = rng.normal(size=(len(trg), td))
        out = out0.copy()
        if uk < 0:
            with pytest.raises(S.StkError):
                S.evaluate_kernel(kernel, p2p, src, np.zeros((len(src), 3)), trg, out, prec)
            continue
        val = uk_values(rng, uk, len(src))
        S.evaluate_kernel(kernel, p2p, src, val, trg, out, prec)
        ref = O.direct(uk, src, val, trg, out=out0.copy())
        assert rel_l2(out - out0, ref - out0) < TOL[prec]


def test_ker_poten_shims(torch_cuda, L):
    """The pvfmm Ker_t-signature shims accumulate the scaled FP64 kernel sum into k_out."""
    rng = np.random.default_rng(9)
    dp = ctypes.POINTER(ctypes.c_double)
    for uk, name in enumerate(UK_NAMES):
        if 11 <= uk <= 15:  # fused / adjoint micro-kernels have no ker_poten shim
            continue
        src = rng.random((200, 3))
        trg = np.concatenate([src[:20], rng.random((50, 3))])
        val = uk_values(rng, uk, len(src))
        out = rng.normal(size=(len(trg), UK_TDIM[uk]))
        ref = O.direct(uk, src, val, trg, out=out.copy())
        fn = getattr(L, "stk_ker_" + name)
        fn(src.ctypes.data_as(dp), len(src), val.ctypes.data_as(dp), 1, trg.ctypes.data_as(dp), len(trg),
           out.ctypes.data_as(dp), None)
        assert L.stk_ker_last_status() == 0
        assert rel_l2(out, ref) < 1e-12, name
        # dof != 1 is rejected without touching k_out
        before = out.copy()
        fn(src.ctypes.data_as(dp), len(src), val.ctypes.data_as(dp), 2, trg.ctypes.data_as(dp), len(trg),
           out.ctypes.data_as(dp), None)
        assert L.stk_ker_last_status() != 0 and np.array_equal(out, before)


def test_invalid_arguments_fail_loudly(torch_cuda, L):
    assert L.stk_ukernel_direct_device(99, 1, 1, 1, 1, 1, 1, 0, 0) != 0
    assert L.stk_ukernel_direct_device(0, -1, 0, 0, 1, 0, 0, 0, 0) != 0
    assert L.stk_ukernel_direct_device(0, 4, 0, 0, 4, 0, 0, 0, 0) != 0  # null pointers
    assert L.stk_ukernel_direct_device(0, 4, 8, 8, 4, 8, 8, 7, 0) != 0  # bad precision


def test_fp64_rsqrt_pointwise():
    """The FP64 path's reciprocal square root (hardware approximation + one third-order
    step) to within a few ulp of 1/sqrt over 24 decades of r^2: laplace_p of one
    unit charge at the origin against q / (4 pi |r|) per target."""
    import torch
    assert torch.cuda.is_available()
    import stkfmm_b200 as S
    rng = np.random.default_rng(17)
    n = 4000
    dirs = rng.normal(size=(n, 3))
    dirs /= np.linalg.norm(dirs, axis=1)[:, None]
    trg = dirs * np.logspace(-12, 0.2, n)[:, None]
    src = np.zeros((1, 3))
    out = np.zeros((n, 4))
    S.evaluate_kernel(S.KERNEL.LapPGrad, S.PPKERNEL.SLS2T, src, np.ones((1, 1)), trg, out)
    r2 = trg[:, 0] * trg[:, 0] + trg[:, 1] * trg[:, 1] + trg[:, 2] * trg[:, 2]
    ref = 1.0 / np.sqrt(r2) / (4 * np.pi)
    assert np.max(np.abs(out[:, 0] - ref) / ref) < 1e-15
    # the gradient, -r / (4 pi r^3)
    g = -trg / (r2 * np.sqrt(r2))[:, None] / (4 * np.pi)
    assert np.max(np.abs(out[:, 1:] - g) / np.linalg.norm(g, axis=1)[:, None]) < 2e-15
