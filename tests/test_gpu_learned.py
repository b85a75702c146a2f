"""What the trained network gains (learned CLEAN proposals, committed
weights weights/unet_c4.npz, trained by ``learned.py train`` on 20,000
seeded skies of the 256-antenna spiral layout at 1024^2).

On held-out skies (a seed the training never used) the plain pipeline runs
10 Hogbom major cycles of 200 minor cycles; the learned pipeline must reach
that final residual RMS (x 1.01) in fewer major cycles and less total wall
time.  Every accepted proposal is an exact major cycle: the residual the
loop tracks equals the residual imaged afresh from measured - model
visibilities (to rounding, in the inner half of the image).  A network that proposes nothing (zero weights) leaves the
learned loop identical to the plain one (Hogbom as the fallback).
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def imaging(device):
    import learned as L
    img = L.Imaging(device, L.spiral_layout(1024))
    yield img
    img.close()


def test_learned_reaches_plain_rms_in_fewer_cycles(imaging):
    import learned as L
    rows = L.evaluate(imaging, L.load_weights(), skies=4, seed=4242)
    for r in rows:
        assert r["learned_cycles"] is not None, r
        assert r["learned_cycles"] < r["plain_cycles"], r
    t_plain = sum(r["plain_s"] for r in rows)
    t_learned = sum(r["learned_s"] for r in rows)
    assert t_learned * 1.5 < t_plain, (t_learned, t_plain, rows)


def test_learned_at_twice_the_field(device):
    """The same network on 2048^2 images of the layout (same cell, twice the
    field): with the proposal window (the image's outer eighth on each side
    excluded) every sky reaches the plain RMS in fewer cycles, and no
    component is proposed in the outer band.  (Without the window the
    network put about two thirds of its components and half of its flux in
    that band, which holds the taper correction's amplified imaging errors,
    and no sky of 8 reached the target.)"""
    import torch
    import learned as L
    img = L.Imaging(device, L.spiral_layout(2048))
    try:
        rows = L.evaluate(img, L.load_weights(), skies=2, seed=4243)
        for r in rows:
            assert r["learned_cycles"] is not None and r["learned_cycles"] < r["plain_cycles"], r
        dec = L.Deconvolver(img, L.load_weights())
        comps = torch.from_numpy(L.SkySampler(img.G, img.layout.cell, 98).sample()).to(img.dev)
        meas = torch.empty((img.n, 2), dtype=torch.float32, device=img.dev)
        L.measured_vis(img, comps, meas, 1e-4, torch.Generator(device=img.dev).manual_seed(5))
        rms = dec._residual(meas)
        ok, _, _, n = dec._propose(rms)
        assert ok and n > 0
        G, cell = img.G, img.layout.cell
        c = dec.comps[:n].cpu().numpy()
        X, Y = np.rint(c[:, 0] / cell) + G // 2, np.rint(c[:, 1] / cell) + G // 2
        lo, hi = dec.border, G - dec.border
        assert dec.border == G // 8
        assert ((X >= lo) & (X < hi) & (Y >= lo) & (Y < hi)).all()
        dec.close()
    finally:
        img.close()


def test_accepted_proposals_are_exact_major_cycles(imaging):
    import torch
    import learned as L
    dec = L.Deconvolver(imaging, L.load_weights())
    comps = torch.from_numpy(L.SkySampler(imaging.G, imaging.layout.cell, 99).sample()).to(imaging.dev)
    meas = torch.empty((imaging.n, 2), dtype=torch.float32, device=imaging.dev)
    L.measured_vis(imaging, comps, meas, 1e-4, torch.Generator(device=imaging.dev).manual_seed(3))
    rms0, recs = dec.run(meas, 3, learned=True)
    assert recs[0].kind == "learned" and recs[0].rms < 0.5 * rms0
    assert all(b.rms < a.rms for a, b in zip(recs, recs[1:]))
    tracked, fresh, exact = dec.exact_residual(meas)
    G = imaging.G
    inner = (slice(G // 4, 3 * G // 4),) * 2
    a = tracked.view(G, G)[inner].cpu().numpy().astype(np.float64)
    b = fresh.view(G, G)[inner].cpu().numpy().astype(np.float64)
    # the taper correction divides by up to 1e10 near the image edges, which
    # magnifies the float-atomic summation order of the gridder there (two
    # imagings of the same visibilities differ by ~1e-4 over the whole image);
    # inside the inner half the two residuals agree to rounding, which the
    # cancellation of the ~30x larger images they are differences of raises
    # to ~2e-5
    assert np.linalg.norm(a - b) <= 1e-4 * np.linalg.norm(b)
    assert abs(exact - recs[-1].rms) <= 1e-2 * exact, (exact, recs[-1].rms)
    dec.close()


def test_no_proposal_falls_back_to_hogbom(imaging, sdp):
    import torch
    import learned as L
    probe = sdp.UNet(sdp.load(), L.IN_CHANNELS, 1, 8, 8, training=False)
    zeros = np.zeros(probe.num_params, np.float32)
    probe.close()
    dec = L.Deconvolver(imaging, zeros)
    comps = torch.from_numpy(L.SkySampler(imaging.G, imaging.layout.cell, 5).sample()).to(imaging.dev)
    meas = torch.empty((imaging.n, 2), dtype=torch.float32, device=imaging.dev)
    L.measured_vis(imaging, comps, meas, 1e-4, torch.Generator(device=imaging.dev).manual_seed(4))
    _, plain = dec.run(meas, 3, learned=False)
    _, lrn = dec.run(meas, 3, learned=True)
    assert [r.kind for r in lrn] == ["hogbom"] * 3
    for a, b in zip(plain, lrn):
        # same kernels in the same order; the residual RMS differs only by the
        # gridder's float-atomic order magnified at the image edges
        assert abs(a.rms - b.rms) <= 1e-3 * a.rms and a.components == b.components
    dec.close()


@pytest.mark.parametrize("grid", [1024, 2048])
def test_network_on_window_crop_matches_full_image(device, grid):
    """The network runs on the centred crop that holds the proposal window
    plus 64 pixels (offset a multiple of 16): on the same residual image its
    output inside the window, and so the components it proposes, are the
    full-image run's bit for bit.  (The residual is imaged once: imaging
    twice differs in the last bits, the gridder's float atomics.)"""
    import torch
    import learned as L
    img = L.Imaging(device, L.spiral_layout(grid))
    try:
        comps = torch.from_numpy(L.SkySampler(img.G, img.layout.cell, 77).sample()).to(img.dev)
        meas = torch.empty((img.n, 2), dtype=torch.float32, device=img.dev)
        L.measured_vis(img, comps, meas, 1e-4, torch.Generator(device=img.dev).manual_seed(6))
        full = L.Deconvolver(img, L.load_weights(), crop=False)
        crop = L.Deconvolver(img, L.load_weights(), crop=True)
        full._residual(meas)
        crop.residual.copy_(full.residual)
        G, W, off = img.G, crop.W, crop.crop_off
        assert full.W == G and W < G and off % 16 == 0
        got = []
        for dec in (full, crop):
            n = dec._select()
            c = dec.comps[:n].cpu().numpy().copy()
            got.append(c[np.lexsort((c[:, 2], c[:, 1], c[:, 0]))])
        b = full.border
        out_full = full.out.reshape(G, G)[b:G - b, b:G - b]
        out_crop = crop.out.reshape(W, W)[b - off:W - (b - off), b - off:W - (b - off)]
        assert torch.equal(out_full, out_crop)
        assert len(got[0]) == len(got[1]) > 0
        np.testing.assert_array_equal(got[1], got[0])
        full.close()
        crop.close()
    finally:
        img.close()
