"""Learned screening network: a 4-level convolutional U-Net (32 base channels) trained on the
peak-depth and arrival-time maps the solver produces, run on the library's own kernels
(include/hp2d_nn.h): BF16 weights and activations, FP32 accumulation on the tcgen05 tensor
cores, FP32 master weights updated by Adam.

There is no counterpart in the reference (HydroPol2D has no surrogate).  The network
screens ensemble members: an ensemble of independently trained networks predicts each
member's peak-depth map, and members on which the networks disagree by more than a
threshold go back to the solver (``screening``).

Layout: activations NHWC BF16; a 3x3 convolution is ``y[P, Co] = cols[P, Kp] . W[Co, Kp]^T``
with K index (ky*3 + kx)*Ci + ci, computed as an implicit GEMM that reads tap-shifted boxes of
the input through TMA (``nn.conv3x3``) where the shape allows, else as im2col + GEMM; backward
gives ``dx`` as the convolution of dy with the flipped kernel (same two forms) and
``dW = dy^T . cols`` (split-K GEMM over pixels).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import nn


def ceil64(n: int) -> int:
    return (n + 63) // 64 * 64


def unet_spec(base: int = 32, levels: int = 4, in_ch: int = 4, out_ch: int = 2):
    """Convolution layers (name, in channels, out channels, ReLU) in forward order."""
    c = [base * 2 ** lvl for lvl in range(levels)]
    spec = []
    ci = in_ch
    for lvl in range(levels):
        spec.append((f"enc{lvl}a", ci, c[lvl], True))
        spec.append((f"enc{lvl}b", c[lvl], c[lvl], True))
        ci = c[lvl]
    for lvl in range(levels - 2, -1, -1):
        spec.append((f"up{lvl}", c[lvl + 1], c[lvl], True))
        spec.append((f"dec{lvl}a", 2 * c[lvl], c[lvl], True))
        spec.append((f"dec{lvl}b", c[lvl], c[lvl], True))
    spec.append(("head", c[0], out_ch, False))
    return spec


def forward_flops(H: int, W: int, base: int = 32, levels: int = 4, in_ch: int = 4, out_ch: int = 2) -> float:
    """Multiply-adds x 2 of the convolutions of one sample (unpadded K)."""
    f = 0.0
    for name, ci, co, _ in unet_spec(base, levels, in_ch, out_ch):
        lvl = layer_level(name)
        f += 2.0 * (H >> lvl) * (W >> lvl) * 9 * ci * co
    return f


def layer_level(name: str) -> int:
    """Resolution level of a layer of ``unet_spec`` (0 = full resolution)."""
    if name == "head":
        return 0
    if name.startswith("up"):
        return int(name[2:])
    return int(name[3])


class Conv3x3:
    """One 3x3, stride-1, zero-padded convolution (+ bias, optional ReLU)."""

    def __init__(self, name, ci, co, relu, gen: torch.Generator, device):
        self.name, self.ci, self.co, self.relu = name, ci, co, relu
        self.kp, self.kp2 = ceil64(9 * ci), ceil64(9 * co)
        std = math.sqrt((2.0 if relu else 1.0) / (9 * ci))
        W = torch.zeros(co, self.kp)
        W[:, :9 * ci] = torch.randn(co, 9 * ci, generator=gen) * std
        self.W = W.to(device)
        self.b = torch.zeros(co, device=device)
        self.gW = torch.zeros_like(self.W)
        self.gb = torch.zeros_like(self.b)
        self.mW, self.vW = torch.zeros_like(self.W), torch.zeros_like(self.W)
        self.mb, self.vb = torch.zeros_like(self.b), torch.zeros_like(self.b)
        self.W16 = nn.to_bf16(self.W)
        self.zero_ci = torch.zeros(ci, device=device)
        self.x = self.y = None

    def refresh(self):
        nn.to_bf16(self.W, self.W16)

    def forward(self, x: torch.Tensor, keep: bool = True):
        B, H, W, _ = x.shape
        P = B * H * W
        head = self.name == "head"
        y = torch.empty(P, self.co, dtype=torch.float32 if head else torch.bfloat16, device=x.device)
        epi = "f32_bias" if head else ("bf16_bias_relu" if self.relu else "bf16_bias")
        if nn.conv_ok(x.shape):
            nn.conv3x3(x.contiguous(), self.W16, self.co, y, epi, bias=self.b)   # implicit GEMM
        else:
            nn.gemm(nn.im2col3x3(x, self.kp), self.W16, y, epi, bias=self.b)
        if keep:
            self.x, self.y = x, y
        return y.view(B, H, W, self.co)

    def backward(self, dy: torch.Tensor, need_dx: bool = True):
        """dy [B, H, W, co] bf16 (modified in place by the ReLU mask); accumulates gW, gb."""
        x = self.x
        B, H, W, _ = x.shape
        P = B * H * W
        dy2 = dy.reshape(P, self.co)
        if self.relu:
            nn.relu_bwd(self.y, dy2)
        nn.colsum(dy2, self.gb)
        dyT = nn.transpose(dy2)
        colsT = nn.im2col3x3(x, self.kp, transpose=True)
        tiles = -(-self.co // 128) * -(-self.kp // (256 if self.kp > 128 else self.kp))
        split = max(1, min(P // 64, (2 * 148) // max(tiles, 1)))
        nn.gemm(dyT, colsT, self.gW, "f32_atomic", split_k=split)
        if not need_dx:
            return None
        wt = nn.flip3x3(self.W, self.co, self.ci, self.kp, self.kp2)
        dx = torch.empty(P, self.ci, dtype=torch.bfloat16, device=x.device)
        dyv = dy2.view(B, H, W, self.co)
        if nn.conv_ok(dyv.shape):
            nn.conv3x3(dyv, wt, self.ci, dx, "bf16_bias", bias=self.zero_ci)
        else:
            nn.gemm(nn.im2col3x3(dyv, self.kp2), wt, dx, "bf16_bias", bias=self.zero_ci)
        return dx.view(B, H, W, self.ci)


class UNet:
    """The screening network on one GPU.  ``forward`` takes NHWC BF16 inputs [B, H, W, 4]
    (H, W multiples of 2**(levels-1) with B*(H*W >> 2*(levels-1)) a multiple of 64) and
    returns FP32 outputs [B*H*W, 2]."""

    def __init__(self, seed: int = 0, base: int = 32, levels: int = 4, in_ch: int = 4, out_ch: int = 2,
                 device="cuda"):
        g = torch.Generator().manual_seed(seed)
        self.levels = levels
        self.spec = unet_spec(base, levels, in_ch, out_ch)
        self.layers = {name: Conv3x3(name, ci, co, relu, g, device) for name, ci, co, relu in self.spec}
        self.step_count = 0
        self.loss_buf = torch.zeros(1, device=device)

    # ---------------------------------------------------------------- passes
    def forward(self, x: torch.Tensor, keep: bool = True) -> torch.Tensor:
        L = self.layers
        self._pre, self._pool, self._up, self._cat = [], [], [], []
        h = x
        skips = []
        for lvl in range(self.levels):
            h = L[f"enc{lvl}a"].forward(h, keep)
            h = L[f"enc{lvl}b"].forward(h, keep)
            if lvl < self.levels - 1:
                skips.append(h)
                p = nn.maxpool2(h)
                self._pool.append((h, p))
                h = p
        for lvl in range(self.levels - 2, -1, -1):
            u = nn.upsample2(h)
            u = L[f"up{lvl}"].forward(u, keep)
            s = skips[lvl]
            B, H, W, c = u.shape
            cat = torch.empty(B, H, W, 2 * c, dtype=torch.bfloat16, device=u.device)
            nn.copy_channels(u, 0, c, cat, 0)
            nn.copy_channels(s, 0, c, cat, c)
            h = L[f"dec{lvl}a"].forward(cat, keep)
            h = L[f"dec{lvl}b"].forward(h, keep)
        out = L["head"].forward(h, keep)
        return out.reshape(-1, out.shape[-1])

    def backward(self, dout: torch.Tensor, shape):
        """dout [P, out_ch] bf16 = d loss / d output."""
        L = self.layers
        B, H, W = shape
        dh = L["head"].backward(dout.view(B, H, W, -1))
        dskip = [None] * (self.levels - 1)
        for lvl in range(self.levels - 1):
            dh = L[f"dec{lvl}b"].backward(dh)
            dcat = L[f"dec{lvl}a"].backward(dh)
            c = dcat.shape[-1] // 2
            du = torch.empty(dcat.shape[:-1] + (c,), dtype=torch.bfloat16, device=dcat.device)
            ds = torch.empty_like(du)
            nn.copy_channels(dcat, 0, c, du, 0)
            nn.copy_channels(dcat, c, c, ds, 0)
            dskip[lvl] = ds
            du = L[f"up{lvl}"].backward(du)
            dh = nn.upsample2_bwd(du)
        for lvl in range(self.levels - 1, -1, -1):
            if lvl < self.levels - 1:
                pre, post = self._pool[lvl]
                g = dskip[lvl]
                nn.maxpool2_bwd(pre, post, dh, g)   # g += routed gradient
                dh = g
            dh = L[f"enc{lvl}b"].backward(dh)
            dh = L[f"enc{lvl}a"].backward(dh, need_dx=lvl > 0)

    def zero_grad(self):
        for c in self.layers.values():
            c.gW.zero_()
            c.gb.zero_()

    def adam_step(self, lr: float, weight_decay: float = 0.0):
        self.step_count += 1
        for c in self.layers.values():
            nn.adam(c.W, c.gW, c.mW, c.vW, c.W16, lr, self.step_count, weight_decay=weight_decay)
            nn.adam(c.b, c.gb, c.mb, c.vb, None, lr, self.step_count)

    def loss_and_grad(self, x, target, weight):
        """Forward, weighted mean squared error, backward; returns the loss tensor (device)."""
        B, H, W, _ = x.shape
        out = self.forward(x)
        P = out.shape[0]
        nch = target.shape[1]
        self.loss_buf.zero_()
        dout = torch.empty(P, out.shape[1], dtype=torch.bfloat16, device=x.device)
        nn.mse(out, target, weight, 1.0 / (P * nch), self.loss_buf, dout)
        self.zero_grad()
        self.backward(dout, (B, H, W))
        return self.loss_buf

    def train_step(self, x, target, weight, lr, weight_decay=0.0):
        loss = self.loss_and_grad(x, target, weight)
        self.adam_step(lr, weight_decay)
        return loss

    def predict(self, x: torch.Tensor) -> torch.Tensor:
        return self.forward(x, keep=False)

    # ---------------------------------------------------------------- weights
    def state(self) -> dict:
        return {n: (c.W.detach().cpu().numpy().copy(), c.b.detach().cpu().numpy().copy())
                for n, c in self.layers.items()}

    def grads(self) -> dict:
        return {n: (c.gW.detach().cpu().numpy().copy(), c.gb.detach().cpu().numpy().copy())
                for n, c in self.layers.items()}

    def load(self, state: dict):
        for n, (W, b) in state.items():
            c = self.layers[n]
            c.W.copy_(torch.from_numpy(np.asarray(W, dtype=np.float32)))
            c.b.copy_(torch.from_numpy(np.asarray(b, dtype=np.float32)))
            c.refresh()
