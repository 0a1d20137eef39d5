"""The tcgen05 BF16 GEMM (hp2d_nn_gemm) against an FP32 matmul of the same BF16 inputs
(torch on the CPU, TF32 off), over tile edges, every N-tile width, split-K and every
epilogue.  Tolerance: FP32 accumulation in a different order, |err| <= 1e-4 * sqrt(K) *
max|a||b| scale, plus one BF16 rounding of the output for the BF16 epilogues."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _ref(A, B):
    return A.float().cpu() @ B.float().cpu().T


@pytest.mark.parametrize("M,N,K", [(128, 32, 64), (256, 64, 128), (300, 100, 192), (512, 128, 576),
                                   (128, 256, 3456), (1000, 320, 320), (64, 48, 64)])
def test_gemm_f32(M, N, K):
    from hydropol2d_b200 import nn
    g = torch.Generator().manual_seed(M * 7 + N)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
    Cg = torch.full((M, N), float("nan"), device="cuda")
    nn.gemm(A, B, Cg, "f32")
    nn.check()
    ref = _ref(A, B)
    err = (Cg.cpu() - ref).abs().max().item()
    assert err <= 1e-4 * np.sqrt(K) * 4, err


def test_gemm_split_k_atomic():
    from hydropol2d_b200 import nn
    g = torch.Generator().manual_seed(3)
    M, N, K = 64, 320, 64 * 40
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
    Cg = torch.ones((M, N), device="cuda")
    nn.gemm(A, B, Cg, "f32_atomic", split_k=7)
    nn.check()
    ref = _ref(A, B) + 1.0
    err = (Cg.cpu() - ref).abs().max().item()
    assert err <= 1e-4 * np.sqrt(K) * 4, err


@pytest.mark.parametrize("epi", ["bf16_bias_relu", "bf16_bias", "f32_bias"])
def test_gemm_bias_epilogues(epi):
    from hydropol2d_b200 import nn
    g = torch.Generator().manual_seed(5)
    M, N, K = 384, 96, 256
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
    bias = torch.randn(N, generator=g).cuda()
    dt = torch.float32 if epi == "f32_bias" else torch.bfloat16
    Cg = torch.zeros((M, N), dtype=dt, device="cuda")
    nn.gemm(A, B, Cg, epi, bias=bias)
    nn.check()
    ref = _ref(A, B) + bias.cpu()
    if epi == "bf16_bias_relu":
        ref = ref.clamp_min(0)
    got = Cg.float().cpu()
    tol = 1e-4 * np.sqrt(K) * 4 + (ref.abs() * 2 ** -8 if dt == torch.bfloat16 else 0)
    assert bool(((got - ref).abs() <= tol).all()), (got - ref).abs().max().item()


def test_gemm_rejects_bad_shapes():
    from hydropol2d_b200 import HP2DError, nn
    A = torch.zeros(128, 100, dtype=torch.bfloat16, device="cuda")
    B = torch.zeros(32, 100, dtype=torch.bfloat16, device="cuda")
    C = torch.zeros(128, 32, device="cuda")
    with pytest.raises(HP2DError):
        nn.gemm(A, B, C)   # K not a multiple of 64
