"""The tensor-core BF16 GEMM of the learned closure (nse2d_gemm_bf16: tcgen05.mma with the
accumulator in tensor memory) against a plain PyTorch FP32 matmul of the same BF16 values.

Both sides multiply exactly representable BF16 numbers and accumulate in FP32, in different
orders, so the bar is a few FP32 ulps of the sum of |a_k b_k|: 1e-5 of it per element.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [(128, 16, 64), (256, 32, 320), (384, 48, 128), (1024, 256, 128), (33024, 32, 320), (640, 128, 640)]


@pytest.mark.parametrize("M,N,K", CASES)
def test_gemm_matches_fp32(nse, cuda, M, N, K):
    torch = cuda
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn((M, K), device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn((N, K), device="cuda", generator=g).to(torch.bfloat16)
    Cf, _ = nse.gemm_bf16(A, B)
    ref = A.float() @ B.float().T
    scale = A.float().abs() @ B.float().abs().T
    err = ((Cf - ref).abs() / (scale + 1e-30)).max().item()
    assert err < 1e-5, err


def test_gemm_bias_relu_bf16(nse, cuda):
    torch = cuda
    g = torch.Generator(device="cuda").manual_seed(7)
    M, N, K = 512, 64, 192
    A = torch.randn((M, K), device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn((N, K), device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn((N,), device="cuda", generator=g)
    Cf, Cb = nse.gemm_bf16(A, B, bias=bias, relu=True, out_f32=True, out_bf16=True)
    ref = A.float() @ B.float().T + bias
    scale = A.float().abs() @ B.float().abs().T + bias.abs()
    assert ((Cf - ref).abs() / scale).max().item() < 1e-5
    # the BF16 output is ReLU(C) rounded to nearest
    assert torch.equal(Cb, torch.relu(Cf).to(torch.bfloat16))


def test_gemm_rejects_bad_shapes(nse, cuda):
    torch = cuda
    A = torch.zeros((100, 64), device="cuda", dtype=torch.bfloat16)
    B = torch.zeros((16, 64), device="cuda", dtype=torch.bfloat16)
    with pytest.raises(nse.Nse2dError):
        nse.gemm_bf16(A, B)
