"""Python handles on the learned screening network's kernels (include/hp2d_nn.h).

Device memory comes from torch tensors (plumbing only: every computation below is one of
the library's own kernels).  BF16 tensors are torch.bfloat16; their bits cross the C ABI as
uint16.  Calls run on torch's current CUDA stream, so they can be captured in a CUDA graph.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _abi

EPI = _abi.NN_EPI


def _L():
    return _abi.lib()


def _p(t: torch.Tensor | None):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ok(st: int):
    if st != 0:
        raise _abi.HP2DError(st, _L().hp2d_nn_error().decode())


def check():
    """Synchronises and raises if a GEMM wait ran out (the kernels' error flag)."""
    _ok(_L().hp2d_nn_check())


def gemm(A: torch.Tensor, B: torch.Tensor, C_out: torch.Tensor, epilogue: str = "f32",
         bias: torch.Tensor | None = None, split_k: int = 1, M: int | None = None, N: int | None = None,
         K: int | None = None):
    """C_out (epilogue) A[M, K] B[N, K]^T with A, B bf16 K-major (row pitch = stride(0))."""
    M = A.shape[0] if M is None else M
    N = B.shape[0] if N is None else N
    K = A.shape[1] if K is None else K
    assert A.dtype == torch.bfloat16 and B.dtype == torch.bfloat16 and A.stride(1) == 1 and B.stride(1) == 1
    assert C_out.stride(1) == 1
    _ok(_L().hp2d_nn_gemm(M, N, K, _p(A), A.stride(0), _p(B), B.stride(0), _p(C_out), C_out.stride(0),
                          _p(bias), EPI[epilogue], int(split_k), _stream()))


def conv_ok(x_shape) -> bool:
    """Whether ``conv3x3`` (implicit GEMM) takes an NHWC input of this shape."""
    _, H, W, Cc = x_shape
    rows_ok = W % 128 == 0 or (128 % W == 0 and H % (128 // W) == 0)
    return Cc >= 32 and Cc % 32 == 0 and rows_ok and (H * W) % 128 == 0


def conv3x3(x: torch.Tensor, w16: torch.Tensor, Co: int, out: torch.Tensor, epilogue: str,
            bias: torch.Tensor | None = None):
    """out[P, Co] (epilogue) = 3x3 convolution of x [B, H, W, C] with w16 [Co, >= 9C] (bf16,
    K index (ky*3 + kx)*C + c), as an implicit GEMM (no im2col buffer)."""
    Bn, H, W, Cc = x.shape
    assert x.is_contiguous() and w16.stride(1) == 1 and out.stride(1) == 1
    _ok(_L().hp2d_nn_conv3x3(_p(x), Bn, H, W, Cc, _p(w16), w16.stride(0), Co, _p(bias), _p(out), out.stride(0),
                             EPI[epilogue], _stream()))


def im2col3x3(x: torch.Tensor, Kp: int, transpose: bool = False, out: torch.Tensor | None = None):
    Bn, H, W, Cc = x.shape
    P = Bn * H * W
    if out is None:
        out = torch.empty((Kp, P) if transpose else (P, Kp), dtype=torch.bfloat16, device=x.device)
    _ok(_L().hp2d_nn_im2col3x3(_p(x), Bn, H, W, Cc, _p(out), Kp, int(transpose), _stream()))
    return out


def transpose(x: torch.Tensor, out: torch.Tensor | None = None):
    rows, cols = x.shape
    if out is None:
        out = torch.empty((cols, rows), dtype=x.dtype, device=x.device)
    _ok(_L().hp2d_nn_transpose(_p(x), rows, cols, x.stride(0), _p(out), out.stride(0), _stream()))
    return out


def maxpool2(x: torch.Tensor):
    Bn, H, W, Cc = x.shape
    y = torch.empty((Bn, H // 2, W // 2, Cc), dtype=x.dtype, device=x.device)
    _ok(_L().hp2d_nn_maxpool2(_p(x), Bn, H, W, Cc, _p(y), _stream()))
    return y


def maxpool2_bwd(x, y, dy, dx=None):
    """Gradient of 2x2 max pooling; with ``dx`` given it is added to ``dx`` in place."""
    Bn, H, W, Cc = x.shape
    acc = dx is not None
    if dx is None:
        dx = torch.empty_like(x)
    _ok(_L().hp2d_nn_maxpool2_bwd(_p(x), _p(y), _p(dy), Bn, H, W, Cc, _p(dx), int(acc), _stream()))
    return dx


def upsample2(x):
    Bn, H, W, Cc = x.shape
    y = torch.empty((Bn, 2 * H, 2 * W, Cc), dtype=x.dtype, device=x.device)
    _ok(_L().hp2d_nn_upsample2(_p(x), Bn, H, W, Cc, _p(y), _stream()))
    return y


def upsample2_bwd(dy):
    Bn, H2, W2, Cc = dy.shape
    dx = torch.empty((Bn, H2 // 2, W2 // 2, Cc), dtype=dy.dtype, device=dy.device)
    _ok(_L().hp2d_nn_upsample2_bwd(_p(dy), Bn, H2 // 2, W2 // 2, Cc, _p(dx), _stream()))
    return dx


def copy_channels(src, c0, n, dst, o0):
    P = src.numel() // src.shape[-1]
    _ok(_L().hp2d_nn_copy_channels(_p(src), src.shape[-1], c0, n, P, _p(dst), dst.shape[-1], o0, _stream()))


def relu_bwd(y, dy):
    _ok(_L().hp2d_nn_relu_bwd(_p(y), _p(dy), y.numel(), _stream()))


def colsum(dz2d, out):
    P, Cc = dz2d.shape
    _ok(_L().hp2d_nn_colsum(_p(dz2d), P, Cc, dz2d.stride(0), _p(out), _stream()))


def mse(pred, target, weight, scale, loss, dpred):
    P = target.shape[0]
    nch = target.shape[1]
    _ok(_L().hp2d_nn_mse(_p(pred), pred.stride(0), _p(target), _p(weight), P, nch, float(scale), _p(loss),
                         _p(dpred), dpred.stride(0), _stream()))


def adam(w, g, m, v, w_bf16, lr, step, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
    _ok(_L().hp2d_nn_adam(_p(w), _p(g), _p(m), _p(v), _p(w_bf16), w.numel(), float(lr), float(beta1),
                          float(beta2), float(eps), float(weight_decay), int(step), _stream()))


def flip3x3(w, Co, Ci, Kp, Kp2, out=None):
    if out is None:
        out = torch.empty((Ci, Kp2), dtype=torch.bfloat16, device=w.device)
    _ok(_L().hp2d_nn_flip3x3(_p(w), Co, Ci, Kp, _p(out), Kp2, _stream()))
    return out


def to_bf16(x, out=None):
    if out is None:
        out = torch.empty(x.shape, dtype=torch.bfloat16, device=x.device)
    _ok(_L().hp2d_nn_f32_to_bf16(_p(x), _p(out), x.numel(), _stream()))
    return out
