"""The oracle's FFT (behind the FFTW-API shim) against numpy.fft (pocketfft):
FFTW_FORWARD = exp(-2 pi i ...), FFTW_BACKWARD = exp(+2 pi i ...) without
normalisation, i.e. numpy's ifft2 times N0 * N1."""
from __future__ import annotations

import numpy as np
import pytest


@pytest.mark.parametrize("G", [8, 16, 64, 256, 12, 36])
def test_fft_matches_numpy(oracle64, G):
    rng = np.random.default_rng(G)
    x = rng.standard_normal((G, G)) + 1j * rng.standard_normal((G, G))
    pairs = np.stack([x.real, x.imag], -1).reshape(-1, 2)
    fwd = oracle64.fft2d(G, pairs, -1)
    inv = oracle64.fft2d(G, pairs, +1)
    ref_f = np.fft.fft2(x)
    ref_i = np.fft.ifft2(x) * G * G
    got_f = (fwd[:, 0] + 1j * fwd[:, 1]).reshape(G, G)
    got_i = (inv[:, 0] + 1j * inv[:, 1]).reshape(G, G)
    assert np.abs(got_f - ref_f).max() <= 1e-10 * np.abs(ref_f).max()
    assert np.abs(got_i - ref_i).max() <= 1e-10 * np.abs(ref_i).max()


def test_fft_round_trip_scales_by_n(oracle64):
    G = 32
    x = np.random.default_rng(1).standard_normal((G * G, 2))
    back = oracle64.fft2d(G, oracle64.fft2d(G, x, -1), +1)
    np.testing.assert_allclose(back, x * G * G, rtol=0, atol=1e-9)


def test_point_source_fft_is_flat(oracle64):
    """A delta at the origin transforms to a constant (known answer)."""
    G = 16
    x = np.zeros((G * G, 2))
    x[0, 0] = 1.0
    out = oracle64.fft2d(G, x, -1)
    np.testing.assert_allclose(out[:, 0], 1.0, atol=1e-15)
    np.testing.assert_allclose(out[:, 1], 0.0, atol=1e-15)
