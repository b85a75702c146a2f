"""Learned-proposal U-Net on the GPU against its CPU oracle (oracle/unet_ref.py).

* forward output (with and without the per-image scale) within 5e-3
  relative L2 of the oracle, whose BF16 rounding points are the device's;
* parameter gradients of every layer within 1e-2 relative L2 on networks
  whose relus are on or off by a wide margin (same masks on both sides; the
  device sums in FP32 in another order, so a BF16 rounding can land one ulp
  apart), and within 0.25 (cosine >= 0.99 overall) on an He-initialised
  network, where a pre-activation within rounding of zero can take the
  other mask; gradients of the padded input channels exactly zero;
* the blurred squared-error loss and its gradient (FP32 against float64);
* Adam against a float32 restatement, over two steps;
* a few optimiser steps on one batch lower the loss (the training path runs
  end to end).
The convolutions run on the tcgen05 path (the default); the mma.sync path
is compared with it.  Sizes cover partial tiles at every level (24 x 40:
the deepest level is 3 x 5) and, at 3 x 256 x 256, several tiles per row,
64-channel chunks and the two output-channel slices of the 384-channel data
gradient; widths divisible by 16 take the shared staged input of the
32/64-channel layers (16 x 16: one partial tile; 40 x 384: three tiles per
row at the top level, partial tile rows, tile edges inside the image).
"""
from __future__ import annotations

import numpy as np
import pytest

import unet_ref as U
from conftest import rel_rms

pytestmark = pytest.mark.gpu


def _setup(sdp, n, c, h, w, seed, training=True):
    import torch
    rng = np.random.default_rng(seed)
    p = U.init_params(32, c, rng)
    layers, head, total = U.layer_table(32)
    for cin, cout, wo, bo in layers:
        p[bo:bo + cout] = (0.05 * rng.standard_normal(cout)).astype(np.float32)
    p[head[1]] = 0.01
    net = sdp.UNet(sdp.load(), c, n, h, w, training=training)
    assert net.num_params == total
    for k, (cin, cout, wo, bo) in enumerate(layers):
        assert net.layer(k) == (cin, cout, wo, bo)
    assert net.layer(14)[2:] == head
    net.set_params(p)
    x = rng.standard_normal((n, c, h, w)).astype(np.float32)
    return net, p, x, torch.from_numpy(x).cuda(), rng


@pytest.mark.parametrize("n,c,h,w", [(2, 3, 24, 40), (1, 1, 16, 16), (2, 3, 40, 384)])
def test_forward_matches_oracle(sdp, device, n, c, h, w):
    import torch
    net, p, x, xd, rng = _setup(sdp, n, c, h, w, 11 + h)
    out = torch.empty((n, h, w), dtype=torch.float32, device="cuda")
    net.forward(xd, out)
    net.check()
    ref = U.UNetRef(p, 32, c).forward(x).detach().numpy()
    assert rel_rms(out.cpu().numpy(), ref) <= 5e-3
    scale = np.array([2.5, 0.125][:n], np.float32)
    net.forward(xd, out, scale=torch.from_numpy(scale).cuda())
    ref = U.UNetRef(p, 32, c).forward(x, scale=scale).detach().numpy()
    assert rel_rms(out.cpu().numpy(), ref) <= 5e-3
    net.close()


def _grad_check(sdp, n, c, h, w, seed, margin):
    """Per-layer relative L2 errors of the device gradients against the
    oracle's.  margin: biases of +-20 (random signs per channel) and weights
    at 5% of He scale, so every relu is on or off by a wide margin and the
    device and the oracle use the same masks (the forward passes differ by
    BF16 rounding, which can flip a relu whose input is near zero)."""
    import torch
    net, p, x, xd, rng = _setup(sdp, n, c, h, w, seed)
    layers, head, total = U.layer_table(32)
    if margin:
        for cin, cout, wo, bo in layers:
            p[wo:bo] *= 0.05
            p[bo:bo + cout] = np.where(rng.random(cout) < 0.5, 20.0, -20.0).astype(np.float32)
        net.set_params(p)
    out = torch.empty((n, h, w), dtype=torch.float32, device="cuda")
    net.forward(xd, out)
    ref_net = U.UNetRef(p, 32, c)
    ref_out = ref_net.forward(x)
    gout = rng.standard_normal((n, h, w)).astype(np.float32)
    net.zero_grads()
    net.backward(torch.from_numpy(gout).cuda())
    net.check()
    g = net.get_grads()
    gr = ref_net.grads(ref_out, gout)
    errs = {}
    for k, (cin, cout, wo, bo) in enumerate(layers):
        gw = g[wo:bo].reshape(9, cout, cin)
        rw = gr[wo:bo].reshape(9, cout, cin)
        if k == 0:
            assert not np.any(gw[:, :, c:]), "padded input channels got a gradient"
            gw, rw = gw[:, :, :c], rw[:, :, :c]
        errs[f"w{k}"] = rel_rms(gw, rw)
        errs[f"b{k}"] = rel_rms(g[bo:bo + cout], gr[bo:bo + cout])
    errs["head"] = rel_rms(g[head[0]:], gr[head[0]:])
    cos = float(g.astype(np.float64) @ gr / (np.linalg.norm(g) * np.linalg.norm(gr)))
    net.close()
    return errs, cos


@pytest.mark.parametrize("n,c,h,w,seed", [(2, 3, 24, 40, 21), (3, 3, 256, 256, 22)])
def test_gradients_match_oracle(sdp, device, n, c, h, w, seed):
    errs, cos = _grad_check(sdp, n, c, h, w, seed, margin=True)
    assert max(errs.values()) <= 1e-2, errs
    assert cos >= 0.9999


def test_gradients_random_network(sdp, device):
    """He-initialised network: relu masks can differ where a pre-activation is
    within BF16 rounding of zero, so the bound is loose; the direction of the
    whole gradient still agrees."""
    errs, cos = _grad_check(sdp, 2, 3, 24, 40, 23, margin=False)
    assert max(errs.values()) <= 0.25, errs
    assert cos >= 0.99, (cos, errs)


def test_blur_mse_matches_oracle(sdp, device):
    import torch
    rng = np.random.default_rng(9)
    pred = rng.standard_normal((2, 24, 40)).astype(np.float32)
    tgt = rng.standard_normal((2, 24, 40)).astype(np.float32)
    pd, td = torch.from_numpy(pred).cuda(), torch.from_numpy(tgt).cuda()
    scratch = torch.empty(2 * pred.size, dtype=torch.float32, device="cuda")
    grad = torch.empty_like(pd)
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    device.blur_mse(pd, td, scratch, grad, loss)
    l_ref, g_ref = U.blur_mse(pred, tgt)
    assert abs(float(loss.item()) - l_ref) <= 1e-6 * l_ref
    assert rel_rms(grad.cpu().numpy(), g_ref) <= 1e-6


def test_adam_matches_reference(sdp, device):
    import torch
    n, c, h, w = 1, 2, 16, 32
    net, p, x, xd, rng = _setup(sdp, n, c, h, w, 31)
    out = torch.empty((n, h, w), dtype=torch.float32, device="cuda")
    wts, m, v = p.copy(), np.zeros_like(p), np.zeros_like(p)
    for step in (1, 2):
        net.forward(xd, out)
        net.zero_grads()
        net.backward(torch.from_numpy(rng.standard_normal((n, h, w)).astype(np.float32)).cuda())
        g = net.get_grads()
        net.adam_step(1e-3, 0.9, 0.999, 1e-8)
        wts, m, v = U.adam(wts, g, m, v, step, 1e-3, 0.9, 0.999, 1e-8)
        got = net.get_params()
        np.testing.assert_allclose(got, wts, rtol=2e-6, atol=1e-9)
    net.close()


def test_training_lowers_loss(sdp, device):
    import torch
    n, c, h, w = 4, 3, 32, 32
    net, p, x, xd, rng = _setup(sdp, n, c, h, w, 41)
    # target: a sparse map the input's first plane points at
    tgt = np.zeros((n, h, w), np.float32)
    for i in range(n):
        ys, xs = rng.integers(2, h - 2, 6), rng.integers(2, w - 2, 6)
        tgt[i, ys, xs] = rng.uniform(0.5, 1.0, 6)
    x[:, 0] = tgt + 0.05 * rng.standard_normal((n, h, w))
    xd = torch.from_numpy(x).cuda()
    td = torch.from_numpy(tgt).cuda()
    out = torch.empty((n, h, w), dtype=torch.float32, device="cuda")
    scratch = torch.empty(2 * tgt.size, dtype=torch.float32, device="cuda")
    grad = torch.empty_like(out)
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    losses = []
    for it in range(60):
        net.forward(xd, out)
        device.blur_mse(out, td, scratch, grad, loss)
        losses.append(float(loss.item()))
        net.zero_grads()
        net.backward(grad)
        net.adam_step(1e-3)
    assert np.isfinite(losses).all()
    assert losses[-1] < 0.3 * losses[0], losses[::10]
    net.close()


@pytest.mark.parametrize("n,c,h,w", [(2, 3, 24, 40), (1, 3, 128, 256), (2, 3, 40, 384)])
def test_tensor_paths_agree(sdp, device, n, c, h, w):
    """tcgen05 (tensor memory, TMA) and mma.sync convolutions: the same network
    gives the same outputs and gradients up to BF16 rounding of
    intermediate activations (different FP32 summation orders)."""
    import torch
    net, p, x, xd, rng = _setup(sdp, n, c, h, w, 51)
    gout = torch.from_numpy(rng.standard_normal((n, h, w)).astype(np.float32)).cuda()
    res = {}
    for tc in (True, False):
        net.set_tensor_path(tc)
        out = torch.empty((n, h, w), dtype=torch.float32, device="cuda")
        net.forward(xd, out)
        net.zero_grads()
        net.backward(gout)
        net.check()
        res[tc] = (out.cpu().numpy(), net.get_grads())
    assert rel_rms(res[True][0], res[False][0]) <= 5e-3
    cos = float(res[True][1].astype(np.float64) @ res[False][1] /
                (np.linalg.norm(res[True][1]) * np.linalg.norm(res[False][1])))
    assert cos >= 0.99
    net.close()


def test_tensor_core_wait_timeout_is_reported_and_recoverable(sdp, device):
    """The failure path of the tcgen05 convolution: with an epilogue wait
    limit of one poll the epilogue gives up before the first accumulator is
    ready; the kernel drains the copies and MMAs it had issued, returns, and
    sdp_unet_check reports SDP_ERR_TIMEOUT.  With the default limit restored
    the same forward pass gives the earlier output bit for bit (the context
    is still usable and the convolutions are deterministic)."""
    import torch
    n, c, h, w = 1, 3, 128, 256
    net, p, x, xd, rng = _setup(sdp, n, c, h, w, 61, training=False)
    ref = torch.empty((n, h, w), dtype=torch.float32, device="cuda")
    net.forward(xd, ref)
    net.check()
    net.set_wait_limit(1)
    out = torch.empty_like(ref)
    net.forward(xd, out)
    with pytest.raises(sdp.SdpError) as e:
        net.check()
    assert e.value.status == sdp.SDP_ERR_TIMEOUT
    net.set_wait_limit(0)
    out.zero_()
    net.forward(xd, out)
    net.check()
    np.testing.assert_array_equal(out.cpu().numpy(), ref.cpu().numpy())
    net.close()
