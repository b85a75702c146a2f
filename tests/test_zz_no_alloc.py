"""sdp_hogbom_noalloc: Hogbom CLEAN for callers that cannot allocate device
memory (a runtime whose memory is all fixed before it starts, or whose device
memory belongs to another allocator).  Its scratch is one fixed device array
per GPU instead of a caller workspace.

Called through the C ABI, twice in a row on the same inputs, it must give
what the allocating entry point sdp_hogbom gives: the same components and
model bit for bit (the tolerance the Hogbom parity tests use), and the same
residual.  Sizes beyond its fixed limit are refused.  This file is collected
last so that a stop at the first failure has already run every other test.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scene(G, rng):
    yy, xx = np.mgrid[0:G, 0:G]
    psf = np.exp(-((xx - G // 2) ** 2 + (yy - G // 2) ** 2) / 5.0)
    psf = (psf / psf.max()).astype(np.float32)
    res = 0.002 * rng.standard_normal((G, G))
    for _ in range(12):
        x0, y0 = rng.integers(2, G - 2, 2)
        res += rng.uniform(0.2, 1.0) * np.roll(np.roll(psf, y0 - G // 2, 0), x0 - G // 2, 1)
    return res.astype(np.float32).reshape(-1), psf.reshape(-1)


def test_noalloc_matches_allocating_hogbom(sdp, device):
    import torch
    dev = torch.device("cuda", 0)
    G, minor, max_src = 256, 150, 200
    res, psf = _scene(G, np.random.default_rng(31))
    params = sdp.CleanParams(G, minor, max_src, 0.1, 1.5, 0.0002, 2.5, 1e-4)
    psf_d = torch.from_numpy(psf).to(dev)

    def run(noalloc: bool):
        r = torch.from_numpy(res.copy()).to(dev)
        m = torch.zeros(G * G, dtype=torch.float32, device=dev)
        s = torch.zeros((max_src, 3), dtype=torch.float32, device=dev)
        c = torch.zeros(1, dtype=torch.int32, device=dev)
        if noalloc:
            device.hogbom_noalloc(params, r, psf_d, m, s, c)
        else:
            ws = torch.empty(device.hogbom_workspace_bytes(G), dtype=torch.uint8, device=dev)
            device.hogbom(params, r, psf_d, m, s, c, ws)
        torch.cuda.synchronize()
        n = int(c.item())
        return n, s[:n].cpu().numpy(), m.cpu().numpy(), r.cpu().numpy()

    n0, s0, m0, r0 = run(False)
    assert n0 > 10
    for _ in range(2):  # two calls in a row share the fixed scratch
        n1, s1, m1, r1 = run(True)
        assert n1 == n0
        np.testing.assert_array_equal(s1, s0)
        np.testing.assert_array_equal(m1, m0)
        np.testing.assert_array_equal(r1, r0)


def test_noalloc_refuses_grid_beyond_limit(sdp, device):
    import torch
    dev = torch.device("cuda", 0)
    G = 4097 + 1  # even, above the 4096 limit
    t = torch.zeros(16, dtype=torch.float32, device=dev)
    c = torch.zeros(1, dtype=torch.int32, device=dev)
    params = sdp.CleanParams(G, 10, 10, 0.1, 1.5, 0.0002, 1.0, 1e-4)
    with pytest.raises(sdp.SdpError) as e:
        device.hogbom_noalloc(params, t, t, t, t, c)
    assert e.value.status == 2
    assert "4096" in str(e.value)
