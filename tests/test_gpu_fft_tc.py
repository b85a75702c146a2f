"""Tensor-core 2-D FFT (BF16 split hi/lo products, FP32 accumulation)
against numpy's complex128 FFT (pocketfft), the same reference the FP32
FFT is checked against: forward (sign -1) and unnormalised inverse (+1),
for every supported size, on random data and on a plane wave (a single
non-zero output).  Bound: 1e-4 relative RMS (the north-star bar for
images); measured ~3e-5.  The FP32 transform stays within 1e-6 on the
same inputs."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_rms

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("G", [1024, 2048, 4096])
@pytest.mark.parametrize("sign", [-1, 1])
def test_fft_tc_random(sdp, device, G, sign):
    import torch
    rng = np.random.default_rng(G + sign)
    x = (rng.standard_normal((G * G, 2))).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    out = torch.empty_like(xd)
    work = torch.empty_like(xd)
    device.fft2d_tc(G, xd, out, sign, work)
    z = (x[:, 0] + 1j * x[:, 1]).astype(np.complex128).reshape(G, G)
    ref = np.fft.fft2(z) if sign < 0 else np.fft.ifft2(z) * (G * G)
    ref = np.stack([ref.real.ravel(), ref.imag.ravel()], axis=1)
    err_tc = rel_rms(out.cpu().numpy(), ref)
    device.fft2d(G, xd, out, sign)
    err_f32 = rel_rms(out.cpu().numpy(), ref)
    assert err_tc <= 1e-4, err_tc
    assert err_f32 <= 1e-6, err_f32


def test_fft_tc_plane_wave(sdp, device):
    import torch
    G = 2048
    ky, kx = 37, 1500
    yy, xx = np.mgrid[0:G, 0:G]
    z = np.exp(2j * np.pi * (ky * yy + kx * xx) / G)
    x = np.stack([z.real.ravel(), z.imag.ravel()], axis=1).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    out, work = torch.empty_like(xd), torch.empty_like(xd)
    device.fft2d_tc(G, xd, out, -1, work)
    o = out.cpu().numpy()
    mag = np.hypot(o[:, 0], o[:, 1]).reshape(G, G)
    assert np.unravel_index(np.argmax(mag), mag.shape) == (ky, kx)
    assert abs(mag[ky, kx] - G * G) <= 1e-4 * G * G
    mag[ky, kx] = 0
    assert mag.max() <= 1e-5 * G * G  # every other bin below 1e-5 of the peak


def test_fft_tc_rejects(sdp, device):
    import torch
    x = torch.zeros((512 * 512, 2), device="cuda")
    with pytest.raises(sdp.SdpError):
        device.fft2d_tc(512, x, x.clone(), -1, x.clone())
    y = torch.zeros((1024 * 1024, 2), device="cuda")
    with pytest.raises(sdp.SdpError):
        device.fft2d_tc(1024, y, y.clone(), -1, y)  # work aliases the input
