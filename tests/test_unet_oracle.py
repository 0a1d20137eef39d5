"""Pins the screening network's oracle (oracle/unet_ref.py): its backward pass in FP64 (no
BF16 rounding) against central finite differences of its own loss, on a small U-Net of the
same structure (3 levels, 4 base channels)."""
import numpy as np

from oracle.unet_ref import RefUNet, bf16, im2col, spec


def _state(sp, rng):
    st = {}
    for n, ci, co, relu in sp:
        kp = -(-9 * ci // 64) * 64
        W = np.zeros((co, kp))
        W[:, :9 * ci] = rng.normal(0, np.sqrt(2.0 / (9 * ci)), (co, 9 * ci))
        st[n] = (W, rng.normal(0, 0.1, co))
    return st


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    sp = spec(base=4, levels=3)
    st = _state(sp, rng)
    B, H, W = 2, 16, 16
    x = rng.normal(size=(B, H, W, 4))
    t = rng.normal(size=(B * H * W, 2))
    w = rng.uniform(0.5, 1.0, size=(B * H * W, 2))

    def loss_of(state):
        net = RefUNet(state, base=4, levels=3, emulate_bf16=False)
        return net.loss_grad(net.forward(x), t, w)[0]

    net = RefUNet(st, base=4, levels=3, emulate_bf16=False)
    out = net.forward(x)
    loss, g = net.loss_grad(out, t, w)
    gW, gb = net.backward(g, (B, H, W))
    h = 1e-6
    checked = 0
    for n, ci, co, relu in sp:
        for _ in range(3):
            i, j = rng.integers(co), rng.integers(9 * ci)
            Wp = {k: (v[0].copy(), v[1].copy()) for k, v in st.items()}
            Wm = {k: (v[0].copy(), v[1].copy()) for k, v in st.items()}
            Wp[n][0][i, j] += h
            Wm[n][0][i, j] -= h
            fd = (loss_of(Wp) - loss_of(Wm)) / (2 * h)
            assert abs(fd - gW[n][i, j]) <= 1e-5 * max(1.0, abs(fd)) + 1e-8, (n, i, j, fd, gW[n][i, j])
            checked += 1
        k = rng.integers(co)
        Bp = {kk: (v[0].copy(), v[1].copy()) for kk, v in st.items()}
        Bm = {kk: (v[0].copy(), v[1].copy()) for kk, v in st.items()}
        Bp[n][1][k] += h
        Bm[n][1][k] -= h
        fd = (loss_of(Bp) - loss_of(Bm)) / (2 * h)
        assert abs(fd - gb[n][k]) <= 1e-5 * max(1.0, abs(fd)) + 1e-8, (n, k, fd, gb[n][k])
        # padding columns of K carry no gradient
        assert np.all(gW[n][:, 9 * ci:] == 0)
    assert checked == 3 * len(sp)


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.00390625, 1.005859375, 1.0078125 + 2 ** -9, -3.14159, 65504.0], dtype=np.float32)
    r = bf16(v)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: even mantissa (1.0) wins
    assert r[1] == np.float32(1.0)
    assert r[2] == np.float32(1.0078125)
    assert np.all(np.abs(r - v) <= np.abs(v) * 2 ** -8)


def test_im2col_layout():
    x = np.arange(2 * 3 * 4 * 5, dtype=np.float64).reshape(2, 3, 4, 5)
    cols = im2col(x, 64)
    # centre tap (4) reproduces the input; tap 0 at (0, 0) is padding
    assert np.array_equal(cols[:, 4 * 5:5 * 5], x.reshape(-1, 5))
    assert np.all(cols[0, 0:5] == 0)
    assert np.all(cols[:, 45:] == 0)
