"""CPU oracle of the learned-proposal U-Net (test infrastructure only).

The reference has no network (its deconvolution is Hogbom,
deconvolution_run.c:197-311), so this oracle restates the device network of
the library (4 levels, base 32 channels, 3x3 convolutions with zero padding,
2x2 mean pooling, nearest upsampling, skip concatenation, 1x1 head) in
torch on the CPU, in float64, with autograd for the gradients.

BF16 storage is emulated where the device stores BF16: every activation
(the packed input, each convolution output after its relu, each pooled
tensor, each concatenation) is rounded to BF16 in the forward pass, and the
gradient arriving at each of them is rounded to BF16 in the backward pass
(the device stores those gradients in BF16).  Weights are the BF16 rounding
of the FP32 master copy with the gradient passed straight through (the
device accumulates the weight gradient of the BF16 weights into the FP32
master gradient).  With round=False the same network runs in plain float64,
for finite-difference checks.

Parameter layout (the C layout, sdp_unet_num_params): per 3x3 layer in the
order e0a e0 e1a e1 e2a e2 e3a e3 d2a d2 d1a d1 d0a d0 the weights
[9][out][in] (tap = 3 (dy + 1) + (dx + 1); layer 0's input padded to 32
channels) then the bias [out]; then the head weights [base] and bias [1].
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

LEVELS = 4
IN_PAD = 32


def layer_table(base: int = 32):
    """[(cin, cout, weight_offset, bias_offset)] for the 14 3x3 layers, then
    the head's (weight_offset, bias_offset) and the total parameter count."""
    shapes = []
    for lv in range(LEVELS):
        shapes.append((IN_PAD if lv == 0 else base << (lv - 1), base << lv))
        shapes.append((base << lv, base << lv))
    for lv in range(LEVELS - 2, -1, -1):
        shapes.append(((base << lv) + (base << (lv + 1)), base << lv))
        shapes.append((base << lv, base << lv))
    out, off = [], 0
    for cin, cout in shapes:
        w = off
        off += 9 * cin * cout
        out.append((cin, cout, w, off))
        off += cout
    head = (off, off + base)
    return out, head, off + base + 1


def init_params(base: int, in_channels: int, rng: np.random.Generator) -> np.ndarray:
    """He-normal 3x3 weights (fan-in = 9 x real input channels), zero biases,
    zero weights on the padded input channels, head ~ N(0, 1/base)."""
    layers, head, n = layer_table(base)
    p = np.zeros(n, np.float32)
    for k, (cin, cout, wo, bo) in enumerate(layers):
        real_in = in_channels if k == 0 else cin
        w = rng.standard_normal((9, cout, cin)) * np.sqrt(2.0 / (9 * real_in))
        if k == 0:
            w[:, :, in_channels:] = 0.0
        p[wo:bo] = w.astype(np.float32).reshape(-1)
    p[head[0]:head[1]] = (rng.standard_normal(base) / np.sqrt(base)).astype(np.float32)
    return p


class _Round(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x):
        return x.to(torch.bfloat16).to(x.dtype)

    @staticmethod
    def backward(ctx, g):
        return g.to(torch.bfloat16).to(g.dtype)


class _Ste(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x):
        return x.to(torch.float32).to(torch.bfloat16).to(x.dtype)

    @staticmethod
    def backward(ctx, g):
        return g


class UNetRef:
    def __init__(self, params: np.ndarray, base: int = 32, in_channels: int = 1, round: bool = True):
        self.base, self.in_ch, self.round = base, in_channels, round
        self.layers, self.head, n = layer_table(base)
        assert params.size == n, (params.size, n)
        self.p = torch.tensor(np.asarray(params, np.float64), requires_grad=True)

    def _r(self, x):
        return _Round.apply(x) if self.round else x

    def _w(self, x):
        return _Ste.apply(x) if self.round else x

    def _conv(self, k, x, relu=True):
        cin, cout, wo, bo = self.layers[k]
        w = self._w(self.p[wo:bo]).reshape(3, 3, cout, cin).permute(2, 3, 0, 1)
        y = F.conv2d(x, w, self.p[bo:bo + cout], padding=1)
        return F.relu(y) if relu else y

    def forward(self, x: np.ndarray | torch.Tensor, scale=None) -> torch.Tensor:
        """x: [n][in_channels][h][w]; scale: [n] or None.  Returns [n][h][w]."""
        x = torch.as_tensor(np.asarray(x, np.float64))
        n, c, h, w = x.shape
        if scale is not None:
            s = torch.as_tensor(np.asarray(scale, np.float32)).to(torch.float64)
            x = (x.to(torch.float32) * (1.0 / s.to(torch.float32))[:, None, None, None]).to(torch.float64)
        pad = torch.zeros((n, IN_PAD - c, h, w), dtype=torch.float64)
        x = self._r(torch.cat([x, pad], dim=1))
        e = []
        cur = x
        for lv in range(LEVELS):
            if lv > 0:
                cur = self._r(F.avg_pool2d(e[-1], 2))
            a = self._r(self._conv(2 * lv, cur))
            e.append(self._r(self._conv(2 * lv + 1, a)))
        low = e[-1]
        for lv in range(LEVELS - 2, -1, -1):
            k = 8 + 2 * (LEVELS - 2 - lv)
            cat = self._r(torch.cat([e[lv], F.interpolate(low, scale_factor=2, mode="nearest")], dim=1))
            a = self._r(self._conv(k, cat))
            low = self._r(self._conv(k + 1, a))
        hw = self._w(self.p[self.head[0]:self.head[1]])
        out = torch.einsum("nchw,c->nhw", low, hw) + self.p[self.head[1]]
        if scale is not None:
            out = out * s[:, None, None]
        return out

    def grads(self, out: torch.Tensor, grad_out: np.ndarray) -> np.ndarray:
        """d(sum(out * grad_out))/d(params) as float64."""
        g = torch.as_tensor(np.asarray(grad_out, np.float64))
        (gp,) = torch.autograd.grad(out, self.p, grad_outputs=g)
        return gp.detach().numpy()


def blur_mse(pred: np.ndarray, target: np.ndarray):
    """loss = mean((b * (pred - target))^2), b the 3x3 binomial kernel
    (1 2 1)^T (1 2 1) / 16 with zero padding; returns (loss, d loss / d pred)
    in float64."""
    p = torch.tensor(np.asarray(pred, np.float64), requires_grad=True)
    t = torch.as_tensor(np.asarray(target, np.float64))
    k = torch.tensor([1.0, 2.0, 1.0], dtype=torch.float64)
    k = (k[:, None] * k[None, :] / 16.0)[None, None]
    d = (p - t)[:, None]
    b = F.conv2d(d, k, padding=1)
    loss = (b * b).mean()
    (g,) = torch.autograd.grad(loss, p)
    return float(loss.detach()), g.numpy()


def adam(w, g, m, v, step, lr, b1, b2, eps):
    """One Adam step in float32 (Kingma & Ba 2015, bias-corrected)."""
    w, g, m, v = (np.asarray(a, np.float32).copy() for a in (w, g, m, v))
    c1 = np.float32(1.0 - b1 ** step)
    c2 = np.float32(1.0 - b2 ** step)
    m = np.float32(b1) * m + np.float32(1.0 - b1) * g
    v = np.float32(b2) * v + np.float32(1.0 - b2) * g * g
    w = w - np.float32(lr) * (m / c1) / (np.sqrt(v / c2) + np.float32(eps))
    return w, m, v
