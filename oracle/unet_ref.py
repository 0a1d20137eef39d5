"""Oracle of the learned screening network -- TEST INFRASTRUCTURE ONLY.

A numpy restatement of the U-Net forward pass, loss and backward pass that the GPU kernels
(include/hp2d_nn.h, composed by hydropol2d_b200/surrogate.py) compute.  There is no
counterpart in the reference; this restatement is pinned by central finite differences in
FP64 (tests/test_unet_oracle.py).  With ``emulate_bf16`` it rounds to BF16 at the points
where the GPU path stores BF16 (weights, activations, activation gradients), so the two
agree up to FP32-versus-FP64 accumulation order.

Layers follow ``unet_spec``: (name, in channels, out channels, ReLU); convolution weights
are [Co, Kp] with K index (ky*3 + kx)*Ci + ci and zero columns beyond 9*Ci.
"""
from __future__ import annotations

import numpy as np


def bf16(a) -> np.ndarray:
    """Round-to-nearest-even to BF16, returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def spec(base=32, levels=4, in_ch=4, out_ch=2):
    c = [base * 2 ** lvl for lvl in range(levels)]
    out = []
    ci = in_ch
    for lvl in range(levels):
        out += [(f"enc{lvl}a", ci, c[lvl], True), (f"enc{lvl}b", c[lvl], c[lvl], True)]
        ci = c[lvl]
    for lvl in range(levels - 2, -1, -1):
        out += [(f"up{lvl}", c[lvl + 1], c[lvl], True), (f"dec{lvl}a", 2 * c[lvl], c[lvl], True),
                (f"dec{lvl}b", c[lvl], c[lvl], True)]
    out.append(("head", c[0], out_ch, False))
    return out


def im2col(x, kp):
    B, H, W, C = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    cols = np.zeros((B * H * W, kp), dtype=x.dtype)
    for tap in range(9):
        ky, kx = divmod(tap, 3)
        cols[:, tap * C:(tap + 1) * C] = xp[:, ky:ky + H, kx:kx + W, :].reshape(-1, C)
    return cols


class RefUNet:
    def __init__(self, state: dict, base=32, levels=4, in_ch=4, out_ch=2, emulate_bf16=True):
        self.levels = levels
        self.spec = spec(base, levels, in_ch, out_ch)
        self.emu = emulate_bf16
        self.W = {n: np.asarray(state[n][0], dtype=np.float64) for n, *_ in self.spec}
        self.b = {n: np.asarray(state[n][1], dtype=np.float64) for n, *_ in self.spec}
        self.meta = {n: (ci, co, relu) for n, ci, co, relu in self.spec}

    def _r(self, a):
        return bf16(a).astype(np.float64) if self.emu else a

    def _w16(self, n):
        return bf16(self.W[n]).astype(np.float64) if self.emu else self.W[n]

    # ---------------------------------------------------------------- layers
    def conv(self, n, x):
        ci, co, relu = self.meta[n]
        kp = self.W[n].shape[1]
        cols = im2col(x, kp)
        y = cols @ self._w16(n).T + self.b[n]
        B, H, W, _ = x.shape
        if n == "head":
            y = y.astype(np.float32).astype(np.float64) if self.emu else y
        else:
            if relu:
                y = np.maximum(y, 0)
            y = self._r(y)
        self.saved[n] = (x, y)
        return y.reshape(B, H, W, co)

    def conv_bwd(self, n, dy, need_dx=True):
        ci, co, relu = self.meta[n]
        x, y = self.saved[n]
        B, H, W, _ = x.shape
        d = dy.reshape(-1, co).copy()
        if relu:
            d[~(y > 0)] = 0
        self.gb[n] = d.sum(axis=0)
        kp = self.W[n].shape[1]
        self.gW[n] = d.T @ im2col(x, kp)
        if not need_dx:
            return None
        kp2 = -(-9 * co // 64) * 64
        wf = np.zeros((ci, kp2))
        Wn = self.W[n]
        for tap in range(9):
            wf[:, tap * co:(tap + 1) * co] = Wn[:, (8 - tap) * ci:(9 - tap) * ci].T
        if self.emu:
            wf = bf16(wf).astype(np.float64)
        dx = im2col(d.reshape(B, H, W, co), kp2) @ wf.T
        return self._r(dx).reshape(B, H, W, ci)

    @staticmethod
    def pool(x):
        B, H, W, C = x.shape
        v = x.reshape(B, H // 2, 2, W // 2, 2, C)
        return v.max(axis=(2, 4))

    def pool_bwd(self, pre, post, dy, acc):
        B, H, W, C = pre.shape
        out = acc.copy()
        routed = np.zeros(post.shape, dtype=bool)
        for dyy, dxx in ((0, 0), (0, 1), (1, 0), (1, 1)):
            sl = pre[:, dyy::2, dxx::2, :]
            hit = (~routed) & (sl == post)
            cur = out[:, dyy::2, dxx::2, :]
            if self.emu:
                s = bf16(cur.astype(np.float32) + dy.astype(np.float32)).astype(np.float64)
            else:
                s = cur + dy
            out[:, dyy::2, dxx::2, :] = np.where(hit, s, cur)
            routed |= hit
        return out

    @staticmethod
    def up(x):
        return x.repeat(2, axis=1).repeat(2, axis=2)

    def up_bwd(self, dy):
        f = dy.astype(np.float32) if self.emu else dy
        s = (f[:, 0::2, 0::2] + f[:, 0::2, 1::2]) + (f[:, 1::2, 0::2] + f[:, 1::2, 1::2])
        return self._r(s) if self.emu else s

    # ---------------------------------------------------------------- passes
    def forward(self, x):
        self.saved = {}
        self.pools = []
        h = np.asarray(x, dtype=np.float64)
        skips = []
        for lvl in range(self.levels):
            h = self.conv(f"enc{lvl}a", h)
            h = self.conv(f"enc{lvl}b", h)
            if lvl < self.levels - 1:
                skips.append(h)
                p = self.pool(h)
                self.pools.append((h, p))
                h = p
        for lvl in range(self.levels - 2, -1, -1):
            u = self.conv(f"up{lvl}", self.up(h))
            h = self.conv(f"dec{lvl}a", np.concatenate([u, skips[lvl]], axis=-1))
            h = self.conv(f"dec{lvl}b", h)
        out = self.conv("head", h)
        return out.reshape(-1, out.shape[-1])

    def loss_grad(self, out, target, weight):
        """Weighted mean squared error and d loss / d out (BF16-rounded when emulating)."""
        P, nch = target.shape
        scale = 1.0 / (P * nch)
        if self.emu:
            o32 = out.astype(np.float32)
            d = o32 - target.astype(np.float32)
            w = weight.astype(np.float32)
            loss = float(np.sum(w.astype(np.float64) * d.astype(np.float64) ** 2) * scale)
            g = ((np.float32(2.0) * w) * d) * np.float32(scale)
            return loss, bf16(g).astype(np.float64)
        d = out - target
        return float(np.sum(weight * d * d) * scale), 2.0 * weight * d * scale

    def backward(self, dout, shape):
        B, H, W = shape
        self.gW, self.gb = {}, {}
        dh = self.conv_bwd("head", dout.reshape(B, H, W, -1))
        dskip = {}
        for lvl in range(self.levels - 1):
            dh = self.conv_bwd(f"dec{lvl}b", dh)
            dcat = self.conv_bwd(f"dec{lvl}a", dh)
            c = dcat.shape[-1] // 2
            dskip[lvl] = dcat[..., c:]
            du = self.conv_bwd(f"up{lvl}", dcat[..., :c].copy())
            dh = self.up_bwd(du)
        for lvl in range(self.levels - 1, -1, -1):
            if lvl < self.levels - 1:
                pre, post = self.pools[lvl]
                dh = self.pool_bwd(pre, post, dh, dskip[lvl])
            dh = self.conv_bwd(f"enc{lvl}b", dh)
            dh = self.conv_bwd(f"enc{lvl}a", dh, need_dx=lvl > 0)
        return self.gW, self.gb
