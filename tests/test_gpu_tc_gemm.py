"""The tcgen05 BF16 GEMM against an FP32 CPU product of the same BF16 inputs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(1, 128, 128, 64), (2, 300, 48, 128), (3, 1000, 32, 384), (1, 77, 256, 192),
                                   (2, 513, 64, 64)])
def test_tc_gemm_matches_cpu(cuda, shape):
    import torch
    from pot3d_b200.tc import check_errors, tc_gemm
    b, M, N, K = shape
    g = torch.Generator().manual_seed(b * 1000 + M)
    A = torch.randn(b, M, K, generator=g).to(torch.bfloat16)
    B = torch.randn(b, N, K, generator=g).to(torch.bfloat16)
    bias = torch.randn(N, generator=g)
    ref = torch.bmm(A.float(), B.float().transpose(1, 2)) + bias
    D = tc_gemm(A.to(cuda), B.to(cuda), bias=bias.to(cuda))
    torch.cuda.synchronize()
    check_errors(cuda)
    got = D.cpu()
    scale = torch.sqrt(torch.tensor(float(K)))
    assert torch.max(torch.abs(got - ref)) <= 1e-4 * scale * 4, torch.max(torch.abs(got - ref))
    Db = tc_gemm(A.to(cuda), B.to(cuda), out_dtype=torch.bfloat16)
    torch.cuda.synchronize()
    ref2 = torch.bmm(A.float(), B.float().transpose(1, 2))
    assert torch.allclose(Db.cpu().float(), ref2, rtol=1e-2, atol=1e-2 * scale)
