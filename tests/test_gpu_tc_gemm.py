"""GPU: the tensor-core GEMM of the mixed M2L (stk_gemm_3xtf32: TF32 tcgen05 products
split into high and low parts, drained per 32-wide K-block into FP32 registers)
against an FP64 torch reference.  FP32 accuracy is the bar: the relative L2 error
stays within a few times that of a plain FP32 GEMM and well below 1e-6, including
ragged sizes (tile edges in M, N and K) and the accumulate form (beta = 1)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


@pytest.mark.parametrize("M,N,K,beta", [(128, 128, 32, 0), (128, 128, 64, 1), (300, 200, 100, 0),
                                        (1000, 777, 240, 1), (636, 2048, 636, 0), (37, 5, 3, 0), (129, 257, 33, 1)])
def test_gemm_3xtf32_fp32_accuracy(torch_cuda, M, N, K, beta):
    from stkfmm_b200 import lib
    torch = torch_cuda
    g = torch.Generator(device="cuda").manual_seed(M + 7 * N + 13 * K)
    lda = K + 1  # a row pitch that is not a multiple of 4: the entry point pads it
    A = torch.randn((M, lda), device="cuda", generator=g, dtype=torch.float32)
    B = torch.randn((N, K), device="cuda", generator=g, dtype=torch.float32)
    C = torch.randn((N, M), device="cuda", generator=g, dtype=torch.float32)  # column-major M x N, ldc = M
    ref = (A[:, :K].double() @ B.double().T).T + (C.double() if beta else 0.0)
    naive = (A[:, :K] @ B.T).T + (C if beta else 0.0)
    rc = lib().stk_gemm_3xtf32(M, N, K, A.data_ptr(), lda, B.data_ptr(), K, C.data_ptr(), M, beta,
                               torch.cuda.current_stream().cuda_stream)
    assert rc == 0, rc
    torch.cuda.synchronize()
    err = float(torch.linalg.norm(C.double() - ref) / torch.linalg.norm(ref))
    err32 = float(torch.linalg.norm(naive.double() - ref) / torch.linalg.norm(ref))
    assert err < max(4 * err32, 1e-7) and err < 1e-6, (err, err32)


def test_gemm_3xtf32_m2l_shape(torch_cuda):
    """The shape of one dense M2L GEMM of the 2M-point RPY PXYZ workload at p = 8
    (level 5): M = k = 636 rows of the stacked factor, N = 4096 boxes of one parity
    type, K = 28672 stacked ranks; operands of ~0.5 GB, larger than L2."""
    from stkfmm_b200 import lib
    torch = torch_cuda
    M, N, K = 636, 4096, 28672
    g = torch.Generator(device="cuda").manual_seed(5)
    A = torch.randn((M, K), device="cuda", generator=g, dtype=torch.float32)
    B = torch.randn((N, K), device="cuda", generator=g, dtype=torch.float32)
    C = torch.zeros((N, M), device="cuda", dtype=torch.float32)
    rc = lib().stk_gemm_3xtf32(M, N, K, A.data_ptr(), K, B.data_ptr(), K, C.data_ptr(), M, 0,
                               torch.cuda.current_stream().cuda_stream)
    assert rc == 0, rc
    torch.cuda.synchronize()
    ref = (A.double() @ B.double().T).T
    naive = (A @ B.T).T
    err = float(torch.linalg.norm(C.double() - ref) / torch.linalg.norm(ref))
    err32 = float(torch.linalg.norm(naive.double() - ref) / torch.linalg.norm(ref))
    assert err < max(4 * err32, 1e-7) and err < 1e-6, (err, err32)
