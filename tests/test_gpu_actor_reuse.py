"""The actors reuse one thread's binning of the visibilities across calls.

std_degridding and std_gridding keep the plan of their last call and reuse
it only when the next call's uvw are equal word for word (checked on the
device), with the same grid size, oversampling, scales, supports and table
length.  These tests change exactly one of those between calls and check that
every result still equals the oracle's, and that the subtract actor's
chunked copies give the exact difference.
"""
from __future__ import annotations

import numpy as np
import pytest

import synth
from conftest import rel_rms

pytestmark = pytest.mark.gpu

GRID_TOL = 2e-6


def _w(seed=31):
    return synth.small_workload(seed=seed, grid_size=128, n_ant=20, n_time=10, num_planes=5, half_support=3,
                                oversampling=16)


def _grid_ref(o, w, uvw, vis, G=128, OS=16, uv_scale=None):
    return o.std_gridding(G, OS, w.gkernels, w.supports, uvw, vis, uv_scale or w.cfg.uv_scale, w.cfg.w_scale)


def test_gridding_reuse_follows_every_input(sdp, actors, oracle32):
    w = _w()
    G, OS = 128, 16
    cfg = sdp.make_config(G, w.cfg.uv_scale, w.cfg.w_scale, OS)
    rng = np.random.default_rng(3)
    uvw = w.uvw.copy()
    # same uvw, new visibilities: the cached binning is reused
    for _ in range(2):
        vis = rng.standard_normal(w.vis.shape).astype(np.float32)
        g = actors.std_gridding(cfg, G, OS, w.gkernels, w.supports, uvw, vis)
        assert rel_rms(g, _grid_ref(oracle32, w, uvw, vis)) <= GRID_TOL
    # one coordinate changed by one ulp-scale step: must not reuse
    uvw2 = uvw.copy()
    uvw2[len(uvw2) // 2, 0] = np.nextafter(uvw2[len(uvw2) // 2, 0], np.float32(1e9))
    uvw2[3, :2] += np.float32(1.5)
    g = actors.std_gridding(cfg, G, OS, w.gkernels, w.supports, uvw2, vis)
    assert rel_rms(g, _grid_ref(oracle32, w, uvw2, vis)) <= GRID_TOL
    # degridding with the same uvw after gridding (shared binning, other tables)
    model = (rng.standard_normal((G * G, 2)) * 1e-2).astype(np.float32)
    actors.set_degrid_mode(sdp.SDP_DEGRID_CONV)
    try:
        p = actors.std_degridding(cfg, G, OS, w.dkernels, w.supports, model, uvw2)
    finally:
        actors.set_degrid_mode(sdp.SDP_DEGRID_NEAREST)
    ref = oracle32.std_degridding(G, OS, w.dkernels, w.supports, model, uvw2, w.cfg.uv_scale, w.cfg.w_scale,
                                  nearest=False)
    assert rel_rms(p, ref) <= GRID_TOL
    # another uv scale with the same uvw: must rebuild
    cfg2 = sdp.make_config(G, w.cfg.uv_scale * 0.9, w.cfg.w_scale, OS)
    g = actors.std_gridding(cfg2, G, OS, w.gkernels, w.supports, uvw2, vis)
    assert rel_rms(g, _grid_ref(oracle32, w, uvw2, vis, uv_scale=w.cfg.uv_scale * 0.9)) <= GRID_TOL
    # fewer visibilities (num_corrected_visibilities): must rebuild
    g = actors.std_gridding(cfg2, G, OS, w.gkernels, w.supports, uvw2, vis, num=len(vis) // 2)
    ref = oracle32.std_gridding(G, OS, w.gkernels, w.supports, uvw2[: len(vis) // 2], vis[: len(vis) // 2],
                                w.cfg.uv_scale * 0.9, w.cfg.w_scale)
    assert rel_rms(g, ref) <= GRID_TOL


def test_subtract_chunks_exact(actors):
    rng = np.random.default_rng(4)
    for n in (0, 1, 3, 1001, 100_003):
        a = rng.standard_normal((n, 2)).astype(np.float32)
        b = rng.standard_normal((n, 2)).astype(np.float32)
        out = actors.subtract_finegrid(a, b)
        np.testing.assert_array_equal(out, a - b)
