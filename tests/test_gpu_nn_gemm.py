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


@pytest.mark.parametrize("B,H,W,C,Co", [(2, 16, 16, 32, 64), (1, 8, 256, 64, 32), (2, 32, 32, 96, 128),
                                        (1, 64, 64, 128, 256), (4, 32, 32, 256, 256), (1, 16, 128, 32, 2)])
def test_implicit_conv_matches_im2col_gemm(B, H, W, C, Co):
    """The implicit-GEMM convolution (4-D TMA boxes shifted per tap, zero fill at the image
    border) against im2col + the same GEMM: identical up to FP32 summation order."""
    from hydropol2d_b200 import nn
    g = torch.Generator().manual_seed(B * 1000 + C + Co)
    x = torch.randn(B, H, W, C, generator=g).to(torch.bfloat16).cuda()
    kp = -(-9 * C // 64) * 64
    w = torch.zeros(Co, kp)
    w[:, :9 * C] = torch.randn(Co, 9 * C, generator=g) * 0.1
    w16 = w.to(torch.bfloat16).cuda()
    bias = torch.randn(Co, generator=g).cuda()
    P = B * H * W
    y_imp = torch.empty(P, Co, device="cuda")
    y_ref = torch.empty(P, Co, device="cuda")
    assert nn.conv_ok(x.shape)
    nn.conv3x3(x, w16, Co, y_imp, "f32_bias", bias=bias)
    nn.gemm(nn.im2col3x3(x, kp), w16, y_ref, "f32_bias", bias=bias)
    nn.check()
    d = (y_imp - y_ref).abs().max().item()
    scale = y_ref.abs().max().item()
    assert d <= 1e-5 * scale + 1e-6, (d, scale)
    yb = torch.empty(P, Co, dtype=torch.bfloat16, device="cuda")
    nn.conv3x3(x, w16, Co, yb, "bf16_bias_relu", bias=bias)
    nn.check()
    ref = y_ref.clamp_min(0)
    assert bool(((yb.float() - ref).abs() <= ref.abs() * 2 ** -8 + 1e-5).all())


@pytest.mark.parametrize("M,N,K,epi,split", [(128 * 400, 64, 192, "f32", 1), (20000, 320, 320, "f32", 1),
                                             (40000, 96, 256, "bf16_bias_relu", 1), (128 * 80, 256, 64 * 12, "f32_atomic", 3),
                                             (60000, 32, 128, "f32_bias", 1)])
def test_persistent_gemm_many_tiles(M, N, K, epi, split):
    """Grids of more tiles than the persistent kernel's resident CTAs run it (two TMEM accumulators, the
    epilogue of one tile overlapping the next): ragged M and N, every epilogue kind, split-K."""
    from hydropol2d_b200 import nn
    g = torch.Generator().manual_seed(M + N + K)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
    bias = torch.randn(N, generator=g).cuda()
    dt = torch.bfloat16 if epi.startswith("bf16") else torch.float32
    C = torch.zeros((M, N), dtype=dt, device="cuda") if epi == "f32_atomic" else \
        torch.full((M, N), float("nan"), dtype=dt, device="cuda")
    if epi == "f32_atomic":
        nn.gemm(A, B, C, epi, split_k=split)
    else:
        nn.gemm(A, B, C, epi, bias=bias if "bias" in epi else None)
    nn.check()
    ref = _ref(A, B)
    if "bias" in epi:
        ref = ref + bias.cpu()
    if epi == "bf16_bias_relu":
        ref = ref.clamp_min(0)
    got = C.float().cpu()
    tol = 1e-4 * np.sqrt(K) * 4 + (ref.abs() * 2 ** -8 if dt == torch.bfloat16 else 0)
    assert bool(((got - ref).abs() <= tol).all()), (got - ref).abs().max().item()


@pytest.mark.parametrize("B,H,W,C,Co", [(4, 128, 128, 32, 64), (4, 128, 128, 64, 128), (2, 128, 256, 32, 32)])
def test_persistent_implicit_conv_against_cpu(B, H, W, C, Co):
    """Implicit convolutions of more tiles than the persistent kernel's resident CTAs (it, per-tile image
    geometry) against a CPU convolution of the same BF16 inputs."""
    from hydropol2d_b200 import nn
    g = torch.Generator().manual_seed(B * H + C)
    x = torch.randn(B, H, W, C, generator=g).to(torch.bfloat16)
    kp = -(-9 * C // 64) * 64
    w = torch.zeros(Co, kp)
    w[:, :9 * C] = torch.randn(Co, 9 * C, generator=g) * 0.1
    w16 = w.to(torch.bfloat16)
    bias = torch.randn(Co, generator=g)
    y = torch.empty(B * H * W, Co, device="cuda")
    nn.conv3x3(x.cuda(), w16.cuda(), Co, y, "f32_bias", bias=bias.cuda())
    nn.check()
    # reference: weights [Co, tap(dy, dx), C] as the library lays them out
    wt = w16.float()[:, :9 * C].reshape(Co, 3, 3, C).permute(0, 3, 1, 2)
    ref = torch.nn.functional.conv2d(x.float().permute(0, 3, 1, 2), wt, bias, padding=1)
    ref = ref.permute(0, 2, 3, 1).reshape(B * H * W, Co)
    d = (y.cpu() - ref).abs().max().item()
    assert d <= 1e-4 * np.sqrt(9 * C) * 4, d
