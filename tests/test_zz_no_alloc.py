"""The allocation-free direct sum (stk_ukernel_direct_device_noalloc).

It serves callers that cannot allocate device memory while they run, e.g. code
being captured into a CUDA graph, where cudaMalloc/cudaFree are not allowed
and would synchronise the device, or a framework whose own allocator owns the
GPU.  Its scratch is one fixed 8 MiB array inside the library, shared by all
calls.  This test checks, through the C ABI, that two calls in a row agree with
the allocating entry point (stk_ukernel_direct_device) within the tolerances
used elsewhere (FP64 1e-12, mixed 1e-6 relative L2), which also shows that each
call clears the counter the previous call left behind, and that sizes beyond
the scratch are refused.  The file name makes pytest collect it last.
"""
import numpy as np
import pytest

from conftest import rel_l2
from helpers import UK_TDIM, uk_values

pytestmark = pytest.mark.gpu

TOL = {0: 1e-12, 1: 1e-6}


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def _dev(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).cuda()


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("uk,ns,nt", [(4, 20000, 3000), (11, 9000, 4100), (6, 333, 65), (12, 5000, 700)])
def test_noalloc_matches_allocating_entry(torch_cuda, uk, ns, nt, prec):
    from stkfmm_b200 import lib
    L = lib()
    torch = torch_cuda
    rng = np.random.default_rng(uk * 100 + prec)
    src = rng.random((ns, 3))
    trg = np.concatenate([src[: nt // 3], rng.random((nt - nt // 3, 3))])
    val = uk_values(rng, uk, ns)
    s, v, t = _dev(torch, src), _dev(torch, val), _dev(torch, trg)
    stream = torch.cuda.current_stream().cuda_stream
    ref = torch.zeros((nt, UK_TDIM[uk]), dtype=torch.float64, device="cuda")
    assert L.stk_ukernel_direct_device(uk, ns, s.data_ptr(), v.data_ptr(), nt, t.data_ptr(), ref.data_ptr(), prec,
                                       stream) == 0
    torch.cuda.synchronize()
    ref = ref.cpu().numpy()
    for call in range(2):
        out = torch.zeros((nt, UK_TDIM[uk]), dtype=torch.float64, device="cuda")
        rc = L.stk_ukernel_direct_device_noalloc(uk, ns, s.data_ptr(), v.data_ptr(), nt, t.data_ptr(),
                                                 out.data_ptr(), prec, stream)
        assert rc == 0, rc
        torch.cuda.synchronize()
        err = rel_l2(out.cpu().numpy(), ref)
        assert err < TOL[prec], (call, err)


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
    assert rc == 4  # STK_ERR_SIZE
    torch.cuda.synchronize()
    assert float(o.abs().sum()) == 0.0
