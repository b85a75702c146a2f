"""The U-Net oracle itself (CPU): parameter layout, and its autograd
gradients against central finite differences in plain float64 (rounding
off), for the network and for the blurred squared-error loss."""
from __future__ import annotations

import numpy as np

import unet_ref as U


def test_layer_table_layout():
    layers, head, n = U.layer_table(32)
    assert [l[:2] for l in layers] == [(32, 32), (32, 32), (32, 64), (64, 64), (64, 128), (128, 128),
                                       (128, 256), (256, 256), (384, 128), (128, 128), (192, 64), (64, 64),
                                       (96, 32), (32, 32)]
    off = 0
    for cin, cout, wo, bo in layers:
        assert wo == off and bo == wo + 9 * cin * cout
        off = bo + cout
    assert head == (off, off + 32) and n == off + 33


def test_network_gradient_finite_differences():
    rng = np.random.default_rng(4)
    p = U.init_params(32, 2, rng).astype(np.float64)
    p[:] += 0.01 * rng.standard_normal(p.size)  # non-zero biases and padded weights
    x = rng.standard_normal((1, 2, 16, 8))
    gout = rng.standard_normal((1, 16, 8))
    net = U.UNetRef(p, 32, 2, round=False)
    g = net.grads(net.forward(x), gout)
    layers, head, n = U.layer_table(32)
    picks = [head[0] + 3, head[1]]
    for cin, cout, wo, bo in layers:
        picks += [int(rng.integers(wo, bo)), int(rng.integers(bo, bo + cout))]

    def f(q):
        return float((U.UNetRef(q, 32, 2, round=False).forward(x).detach().numpy() * gout).sum())

    eps = 1e-6
    for i in picks:
        a, b = p.copy(), p.copy()
        a[i] += eps
        b[i] -= eps
        fd = (f(a) - f(b)) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])


def test_blur_mse_gradient():
    rng = np.random.default_rng(5)
    pred, tgt = rng.standard_normal((2, 6, 9)), rng.standard_normal((2, 6, 9))
    loss, g = U.blur_mse(pred, tgt)
    eps = 1e-6
    for idx in [(0, 0, 0), (1, 5, 8), (0, 3, 4), (1, 0, 7)]:
        a, b = pred.copy(), pred.copy()
        a[idx] += eps
        b[idx] -= eps
        fd = (U.blur_mse(a, tgt)[0] - U.blur_mse(b, tgt)[0]) / (2 * eps)
        assert abs(fd - g[idx]) <= 1e-7 + 1e-6 * abs(fd)
    # direct evaluation of the stencil
    k = np.outer([1, 2, 1], [1, 2, 1]) / 16.0
    d = np.pad(pred - tgt, ((0, 0), (1, 1), (1, 1)))
    b = sum(k[i, j] * d[:, i:i + 6, j:j + 9] for i in range(3) for j in range(3))
    assert abs(loss - float((b * b).mean())) <= 1e-12 * loss


def test_bf16_rounding_points_are_identity_on_bf16_values():
    rng = np.random.default_rng(6)
    p = U.init_params(32, 1, rng)
    x = rng.standard_normal((1, 1, 8, 8))
    a = U.UNetRef(p, 32, 1, round=True).forward(x).detach().numpy()
    b = U.UNetRef(p, 32, 1, round=False).forward(x).detach().numpy()
    # BF16 storage changes the output by a few BF16 ulps at most
    assert np.abs(a - b).max() <= 0.05 * np.abs(b).max()
