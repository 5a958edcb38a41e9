"""The allocation-free direct sum (stk_ukernel_direct_device_noalloc).

It serves callers that cannot allocate device memory while they run: a
framework whose own caching allocator owns the GPU (memory taken behind its
back can make it fail), a program that keeps several streams busy and cannot
afford the device-wide synchronisation of cudaMalloc/cudaFree, or a host that
forbids run-time allocation.  Its scratch is one fixed 8 MiB array inside the
library, shared by all calls.  Through the C ABI this file checks that:

* two calls in a row match the CPU oracle (and the allocating entry point,
  stk_ukernel_direct_device) within the tolerances used elsewhere (FP64 1e-12,
  mixed 1e-6 relative L2), which also shows that each call clears the work
  counter the previous call left behind;
* it takes every micro-kernel the allocating entry point takes without
  per-target values, and refuses the adjoint ones (which need them) with
  STK_ERR_INVALID_ARG;
* a call after warm-up changes neither the device's free memory
  (cudaMemGetInfo) nor torch's allocated bytes;
* sizes beyond the scratch are refused with STK_ERR_SIZE.

The file name makes pytest collect it last.
"""
import numpy as np
import pytest

from conftest import rel_l2
from helpers import UK_TDIM, uk_values
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = {0: 1e-12, 1: 1e-6}
STK_ERR_INVALID_ARG, STK_ERR_SIZE = 1, 4


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def _dev(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _oracle(uk, src, val, trg):
    """The oracle's direct sum; a fused micro-kernel is the sum of its two layers."""
    if uk == 11:  # laplace_pgrad + laplace_dipolepgrad
        return O.direct(1, src, val[:, :1], trg) + O.direct(3, src, val[:, 1:4], trg)
    if uk == 12:  # stokes_pvel + stokes_doublepvel
        return O.direct(9, src, val[:, :4], trg) + O.direct(10, src, val[:, 4:13], trg)
    if uk == 15:  # laplace_p + laplace_dipolep
        return O.direct(0, src, val[:, :1], trg) + O.direct(2, src, val[:, 1:4], trg)
    return O.direct(uk, src, val, trg)


def _inputs(uk, ns, nt, prec):
    rng = np.random.default_rng(uk * 100 + prec)
    src = rng.random((ns, 3))
    trg = np.concatenate([src[: nt // 3], rng.random((nt - nt // 3, 3))])  # coincident points included
    return src, uk_values(rng, uk, ns), trg


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("uk,ns,nt", [(4, 20000, 3000), (11, 9000, 4100), (6, 333, 65), (12, 5000, 700),
                                      (16, 4000, 900), (24, 3000, 500), (27, 2500, 130)])
def test_noalloc_matches_oracle(torch_cuda, uk, ns, nt, prec):
    from stkfmm_b200 import lib
    L = lib()
    torch = torch_cuda
    src, val, trg = _inputs(uk, ns, nt, prec)
    s, v, t = _dev(torch, src), _dev(torch, val), _dev(torch, trg)
    stream = torch.cuda.current_stream().cuda_stream
    ref = _oracle(uk, src, val, trg)
    alloc = torch.zeros((nt, UK_TDIM[uk]), dtype=torch.float64, device="cuda")
    assert L.stk_ukernel_direct_device(uk, ns, s.data_ptr(), v.data_ptr(), nt, t.data_ptr(), alloc.data_ptr(), prec,
                                       stream) == 0
    torch.cuda.synchronize()
    alloc = alloc.cpu().numpy()
    assert rel_l2(alloc, ref) < TOL[prec]
    for call in range(2):
        out = torch.zeros((nt, UK_TDIM[uk]), dtype=torch.float64, device="cuda")
        rc = L.stk_ukernel_direct_device_noalloc(uk, ns, s.data_ptr(), v.data_ptr(), nt, t.data_ptr(),
                                                 out.data_ptr(), prec, stream)
        assert rc == 0, rc
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert rel_l2(got, ref) < TOL[prec], (call, rel_l2(got, ref))
        assert rel_l2(got, alloc) < TOL[prec], (call, rel_l2(got, alloc))


@pytest.mark.parametrize("uk", [13, 14, 29, -1])
def test_noalloc_refuses_kernels_it_cannot_run(torch_cuda, uk):
    """Adjoint micro-kernels need per-target values; ids outside the table do not exist."""
    from stkfmm_b200 import lib
    torch = torch_cuda
    s = torch.zeros((10, 3), dtype=torch.float64, device="cuda")
    v = torch.zeros((10, 4), dtype=torch.float64, device="cuda")
    o = torch.zeros((10, 7), dtype=torch.float64, device="cuda")
    rc = lib().stk_ukernel_direct_device_noalloc(uk, 10, s.data_ptr(), v.data_ptr(), 10, s.data_ptr(), o.data_ptr(),
                                                 0, torch.cuda.current_stream().cuda_stream)
    assert rc == STK_ERR_INVALID_ARG, rc


def _free_bytes():
    import torch
    free, _total = torch.cuda.mem_get_info()  # cudaMemGetInfo
    return free


@pytest.mark.parametrize("prec", [0, 1])
def test_noalloc_allocates_nothing(torch_cuda, prec):
    """After one warm-up call, further calls leave device memory as they found it."""
    from stkfmm_b200 import lib
    L = lib()
    torch = torch_cuda
    uk, ns, nt = 11, 30000, 5000
    src, val, trg = _inputs(uk, ns, nt, prec)
    s, v, t = _dev(torch, src), _dev(torch, val), _dev(torch, trg)
    out = torch.zeros((nt, UK_TDIM[uk]), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    args = (uk, ns, s.data_ptr(), v.data_ptr(), nt, t.data_ptr(), out.data_ptr(), prec, stream)
    assert L.stk_ukernel_direct_device_noalloc(*args) == 0  # warm-up: symbol look-up, occupancy query
    torch.cuda.synchronize()
    free0, torch0 = _free_bytes(), torch.cuda.memory_allocated()
    for _ in range(3):
        assert L.stk_ukernel_direct_device_noalloc(*args) == 0
    torch.cuda.synchronize()
    assert _free_bytes() == free0
    assert torch.cuda.memory_allocated() == torch0
    ref = _oracle(uk, src, val, trg)
    assert rel_l2(out.cpu().numpy(), 4.0 * ref) < TOL[prec]  # four calls accumulated


def test_noalloc_refuses_sizes_beyond_scratch(torch_cuda):
    from stkfmm_b200 import lib
    L = lib()
    torch = torch_cuda
    ns = 200_000  # 200k records of 8 doubles: 12.8 MB > 8 MiB of scratch
    s = torch.zeros((ns, 3), dtype=torch.float64, device="cuda")
    v = torch.zeros((ns, 4), dtype=torch.float64, device="cuda")
    t = torch.zeros((10, 3), dtype=torch.float64, device="cuda")
    o = torch.zeros((10, 4), dtype=torch.float64, device="cuda")
    rc = L.stk_ukernel_direct_device_noalloc(11, ns, s.data_ptr(), v.data_ptr(), 10, t.data_ptr(), o.data_ptr(), 0,
                                             torch.cuda.current_stream().cuda_stream)
    assert rc == STK_ERR_SIZE
    torch.cuda.synchronize()
    assert float(o.abs().sum()) == 0.0
