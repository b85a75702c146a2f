"""Kernels of the learned major cycle against numpy restatements:
input planes, component selection (largest values, whole histogram bins),
FP64 dots and the least-squares step, sky rendering, and the DFT of points
and circular Gaussians (closed-form visibility of a Gaussian)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_rms

pytestmark = pytest.mark.gpu


def test_input_planes(sdp, device):
    import torch
    rng = np.random.default_rng(1)
    G = 96
    r = (rng.standard_normal(G * G) * 3).astype(np.float32)
    psf = rng.standard_normal(G * G).astype(np.float32)
    planes = torch.empty(3 * G * G, dtype=torch.float32, device="cuda")
    s = torch.empty(1, dtype=torch.float32, device="cuda")
    device.unet_input_planes(G, torch.from_numpy(r).cuda(), torch.from_numpy(psf).cuda(), planes, s)
    smax = np.abs(r).max()
    assert float(s.item()) == smax
    got = planes.cpu().numpy().reshape(3, -1)
    v = r * np.float32(1.0 / smax)
    np.testing.assert_allclose(got[0], v, rtol=1e-6, atol=0)
    np.testing.assert_allclose(got[1], np.sign(v) * np.sqrt(np.abs(v)), rtol=1e-6, atol=0)
    np.testing.assert_array_equal(got[2], psf)


@pytest.mark.parametrize("max_count,signed", [(100000, False), (37, False), (1, False), (100000, True), (37, True)])
def test_select_components(sdp, device, max_count, signed):
    import torch
    rng = np.random.default_rng(2 + max_count)
    G, cell, rel = 128, 1.5e-4, 0.05
    prop = (rng.standard_normal(G * G) * 0.02).astype(np.float32)
    idx = rng.choice(G * G, 200, replace=False)
    prop[idx] = rng.uniform(0.01, 1.0, 200).astype(np.float32)
    if signed:
        prop[idx[:60]] *= -1.5
    s = torch.tensor([2.0], dtype=torch.float32, device="cuda")
    comps = torch.zeros((max(max_count, 1), 4), dtype=torch.float32, device="cuda")
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    delta = torch.empty(G * G, dtype=torch.float32, device="cuda")
    ws = device.select_workspace()
    device.select_components(G, cell, torch.from_numpy(prop).cuda(), s, rel, max_count, comps, count, delta, ws,
                             signed=signed)
    n = int(count.item())
    c = comps.cpu().numpy()[:n]
    d = delta.cpu().numpy()
    key = np.abs(prop) if signed else prop
    vmax = key.max()
    lo = np.float32(rel) * vmax
    cand = np.flatnonzero((key >= lo) & (key > 0))
    sel = np.flatnonzero(d != 0)
    assert len(sel) == n <= max_count
    if max_count >= len(cand):
        assert set(sel) == set(cand)
    else:
        # whole bins from the top: every selected value >= every unselected candidate
        rest = np.setdiff1d(cand, sel)
        assert n >= 1 and key[sel].min() >= key[rest].max()
    ys, xs = np.divmod(sel, G)
    exp = {(np.float32((x - G // 2) * cell), np.float32((y - G // 2) * cell), np.float32(2.0) * prop[y * G + x])
           for y, x in zip(ys, xs)}
    got = {(a, b, f) for a, b, f, _ in c}
    assert got == exp


def test_dots_and_step(sdp, device):
    import torch
    rng = np.random.default_rng(3)
    n = 100003
    a = rng.standard_normal(n).astype(np.float32)
    b = (0.3 * a + 0.1 * rng.standard_normal(n)).astype(np.float32)
    dots = torch.empty(2, dtype=torch.float64, device="cuda")
    device.dots(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), dots)
    ab, bb = float(a.astype(np.float64) @ b), float(b.astype(np.float64) @ b)
    d = dots.cpu().numpy()
    assert abs(d[0] - ab) <= 1e-12 * abs(ab) and abs(d[1] - bb) <= 1e-12 * bb
    y = rng.standard_normal(n).astype(np.float32)
    yd = torch.from_numpy(y).cuda()
    alpha = torch.empty(1, dtype=torch.float32, device="cuda")
    device.axpy_ratio(dots, 10.0, torch.from_numpy(b).cuda(), yd, alpha)
    al = np.float32(ab / bb)
    assert float(alpha.item()) == al
    np.testing.assert_allclose(yd.cpu().numpy(), y + al * b, rtol=1e-6, atol=1e-6)
    y2 = yd.cpu().numpy()
    device.axpy_ratio(dots, 1.0, torch.from_numpy(b).cuda(), yd, alpha, sign=-1.0)  # clipped, subtracted
    assert float(alpha.item()) == 1.0
    np.testing.assert_allclose(yd.cpu().numpy(), y2 - b, rtol=1e-6, atol=1e-6)


def test_sky_render(sdp, device):
    import torch
    G, cell = 128, 1e-4
    comps = np.array([[5 * cell, -7 * cell, 0.75, 0.0],
                      [-20 * cell, 11 * cell, 2.0, 2.5 * cell],
                      [30 * cell, 30 * cell, 0.5, 1.0 * cell]], np.float32)
    img = torch.zeros(G * G, dtype=torch.float32, device="cuda")
    device.sky_render(G, cell, torch.from_numpy(comps).cuda(), img)
    im = img.cpu().numpy().reshape(G, G)
    assert im[G // 2 - 7, G // 2 + 5] == np.float32(0.75)
    blob = im[G // 2 + 11 - 12:G // 2 + 11 + 13, G // 2 - 20 - 12:G // 2 - 20 + 13]
    assert abs(blob.sum() - 2.0) <= 2e-3
    assert np.unravel_index(np.argmax(blob), blob.shape) == (12, 12)
    yy, xx = np.mgrid[0:G, 0:G]
    g = 0.5 / (2 * np.pi) * np.exp(-((xx - G // 2 - 30) ** 2 + (yy - G // 2 - 30) ** 2) / 2.0)
    win = (np.abs(xx - G // 2 - 30) <= 4) & (np.abs(yy - G // 2 - 30) <= 4)
    np.testing.assert_allclose(im[win], g[win], rtol=1e-5, atol=1e-7)


def test_dft_gauss(sdp, device):
    import torch
    rng = np.random.default_rng(4)
    n = 5000
    uvw = np.stack([rng.uniform(-3000, 3000, n), rng.uniform(-3000, 3000, n), rng.uniform(-50, 50, n)],
                   axis=1).astype(np.float32)
    src = np.array([[1e-3, -2e-3, 1.0, 0.0], [-4e-3, 5e-4, 0.3, 3e-4], [2e-3, 2e-3, 0.05, 1e-4]], np.float32)
    vis = torch.empty((n, 2), dtype=torch.float32, device="cuda")
    device.dft_gauss(torch.from_numpy(src).cuda(), torch.from_numpy(uvw).cuda(), vis)
    u, v, w = (uvw[:, k].astype(np.float64) for k in range(3))
    l, m, f, sg = (src[:, k].astype(np.float64) for k in range(4))
    h = 0.5 * (l * l + m * m)
    ph = np.outer(u, l) + np.outer(v, m) - np.outer(w, h)
    amp = f / (1 - h) * np.exp(-2 * np.pi ** 2 * np.outer(u * u + v * v, sg * sg))
    ref = (amp * np.exp(-2j * np.pi * ph)).sum(axis=1)
    got = vis.cpu().numpy()
    assert rel_rms(got, np.stack([ref.real, ref.imag], axis=1)) <= 2e-6


def test_dft_pixels(sdp, device):
    """Pixel components against complex128 with the exact positions X cell;
    the fixed-point phase reduction keeps the error near FP32 rounding even
    for long baselines and far pixels (u l up to ~500 cycles here)."""
    import torch
    import learned as L
    lay = L.spiral_layout(2048)
    rng = np.random.default_rng(6)
    uvw = lay.uvw[rng.choice(lay.uvw.shape[0], 20000, replace=False)]
    cell = lay.cell
    X = rng.integers(-1000, 1000, 300)
    Y = rng.integers(-1000, 1000, 300)
    f = rng.uniform(-1, 1, 300)
    comps = np.stack([(X * cell).astype(np.float32), (Y * cell).astype(np.float32), f.astype(np.float32),
                      np.zeros(300, np.float32)], axis=1)
    vis = torch.zeros((uvw.shape[0], 2), dtype=torch.float32, device="cuda")
    uvw_d = torch.from_numpy(uvw).cuda()
    device.dft_pixels(torch.from_numpy(comps).cuda(), cell, uvw_d, vis)
    u, v, w = (uvw[:, k].astype(np.float64) for k in range(3))
    l, m = X * cell, Y * cell
    h = 0.5 * (l * l + m * m)
    ph = np.outer(u, l) + np.outer(v, m) - np.outer(w, h)
    ref = ((f.astype(np.float32).astype(np.float64) / (1 - h)) * np.exp(-2j * np.pi * ph)).sum(axis=1)
    got = vis.cpu().numpy()
    assert rel_rms(got, np.stack([ref.real, ref.imag], axis=1)) <= 3e-6
    # stride 3 (CLEAN components) and accumulation
    c3 = torch.from_numpy(np.ascontiguousarray(comps[:, :3])).cuda()
    device.dft_pixels(c3, cell, uvw_d, vis, accumulate=True)
    assert rel_rms(vis.cpu().numpy(), 2 * np.stack([ref.real, ref.imag], axis=1)) <= 3e-6


@pytest.mark.parametrize("G,border", [(64, 0), (64, 5), (96, 12), (10, 5), (10, 7)])
def test_zero_border(sdp, device, G, border):
    import torch
    rng = np.random.default_rng(G + border)
    img = rng.standard_normal((G, G)).astype(np.float32)
    d = torch.from_numpy(img).cuda()
    device.zero_border(G, border, d)
    exp = img.copy()
    if border > 0:
        exp[:border] = 0
        exp[G - border:] = 0
        exp[:, :border] = 0
        exp[:, G - border:] = 0
    np.testing.assert_array_equal(d.cpu().numpy(), exp)
