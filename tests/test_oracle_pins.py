"""Pins the oracle restatement (oracle/sdp_oracle.c) to the reference.

1. Against the golden fixtures (tests/golden/*.npz), which hold outputs of the
   reference's actors compiled unmodified from their sources
   (tests/golden/make_golden.py): exact equality, float and double builds.
2. When the compiled reference is present (oracle/_ref, built here from the
   reference tree), against it directly on further seeded inputs, including
   the 1229-pixel taper kill at G >= 2460 and a Hogbom run long enough to hit
   the PSF column wrap.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
import synth


def test_wproj_golden_f32(oracle32, golden):
    d = golden("wproj_g64.npz")
    G, OS = int(d["grid_size"]), int(d["oversampling"])
    us, ws = float(d["uv_scale"]), float(d["w_scale"])
    ov, ou, n = oracle32.correct_to_finegrid(G, OS, d["uvw"], d["vis"], us)
    assert n == d["uvw"].shape[0]
    np.testing.assert_array_equal(ou, d["ctf_uvw_f32"])
    np.testing.assert_array_equal(ov, d["ctf_vis_f32"])
    np.testing.assert_array_equal(
        oracle32.std_gridding(G, OS, d["gkernels"], d["supports"], ou, d["vis"], us, ws), d["grid_f32"])
    np.testing.assert_array_equal(
        oracle32.std_gridding(G, OS, d["gkernels"], d["supports"], d["uvw"], d["vis"], us, ws), d["grid_raw_f32"])
    np.testing.assert_array_equal(
        oracle32.std_degridding(G, OS, d["dkernels"], d["supports"], d["model_grid"], ou, us, ws, nearest=True),
        d["degrid_f32"])
    np.testing.assert_array_equal(
        oracle32.std_degridding(G, OS, d["dkernels"], d["supports"], d["model_grid"], d["uvw"], us, ws, nearest=True),
        d["degrid_raw_f32"])
    np.testing.assert_array_equal(oracle32.subtract_vis(d["vis"], d["degrid_f32"]), d["subtract_f32"])
    np.testing.assert_array_equal(
        oracle32.g2g_degridgrid(G, OS, d["gkernels"], d["supports"], d["dkernels"], d["supports"], d["model_grid"],
                                ou, us), d["g2g_f32"])
    np.testing.assert_array_equal(
        oracle32.gridding_cpu(G, 16, d["gkernels"], d["supports"], d["uvw"], d["vis"], us, ws),
        d["gridding_actor_f32"])


def test_wproj_golden_f64(oracle64, golden):
    d = golden("wproj_g64.npz")
    G, OS = int(d["grid_size"]), int(d["oversampling"])
    us, ws = float(d["uv_scale"]), float(d["w_scale"])
    ov, ou, n = oracle64.correct_to_finegrid(G, OS, d["uvw"], d["vis"], us)
    np.testing.assert_array_equal(ou, d["ctf_uvw_f64"])
    np.testing.assert_array_equal(oracle64.std_gridding(G, OS, d["gkernels"], d["supports"], ou, d["vis"], us, ws),
                                  d["grid_f64"])
    np.testing.assert_array_equal(
        oracle64.g2g_degridgrid(G, OS, d["gkernels"], d["supports"], d["dkernels"], d["supports"], d["model_grid"],
                                ou, us), d["g2g_f64"])
    np.testing.assert_array_equal(
        oracle64.gridding_cpu(G, 16, d["gkernels"], d["supports"], d["uvw"], d["vis"], us, ws),
        d["gridding_actor_f64"])


def test_fft_taper_golden(oracle32, oracle64, golden):
    d = golden("fft_g32.npz")
    G = int(d["grid_size"])
    np.testing.assert_array_equal(oracle32.fft2d(G, d["x"], -1), d["fft_fwd_f32"])
    np.testing.assert_array_equal(oracle32.fft2d(G, d["x"], +1), d["fft_inv_f32"])
    np.testing.assert_array_equal(oracle64.fft2d(G, d["x"], -1), d["fft_fwd_f64"])
    np.testing.assert_array_equal(oracle64.fft2d(G, d["x"], +1), d["fft_inv_f64"])
    np.testing.assert_array_equal(oracle32.fft_shift_c2c(G, d["x"]), d["shift_c2c_f32"])
    np.testing.assert_array_equal(oracle32.fft_shift_c2r(G, d["x"]), d["shift_c2r_f32"])
    np.testing.assert_array_equal(oracle32.fft_shift_r2c(G, d["image"]), d["shift_r2c_f32"])
    p = oracle32.half_prolate(G)
    np.testing.assert_array_equal(p, d["prolate_f32"])
    np.testing.assert_array_equal(oracle32.conv_correction(G, d["image"], p), d["taper_f32"])
    np.testing.assert_array_equal(oracle32.merge_grids(G, d["grids4"]), d["merge_f32"])
    np.testing.assert_array_equal(oracle32.subtract_image(G, d["image"], d["image"][::-1].copy()), d["subimg_f32"])


def test_dft_golden(oracle32, oracle64, golden):
    d = golden("dft.npz")
    np.testing.assert_array_equal(oracle32.dft(d["sources"], d["uvw"]), d["vis_f32"])
    np.testing.assert_array_equal(oracle64.dft(d["sources"], d["uvw"]), d["vis_f64"])


def test_hogbom_golden(oracle32, golden):
    d = golden("hogbom_g64.npz")
    G = int(d["grid_size"])
    n, src, model, _ = oracle32.hogbom(G, 100, 200, d["dirty"], d["psf"], float(d["psf_max"]), float(d["cell_size"]))
    assert n == int(d["num_sources"])
    np.testing.assert_array_equal(src, d["sources"])
    np.testing.assert_array_equal(model, d["model"])
    clean, hd = oracle32.clean_psf(G, float(d["psf_max"]), d["psf"])
    np.testing.assert_array_equal(clean, d["clean_psf"])
    np.testing.assert_array_equal(hd, d["halfdims"])


ref_available = pytest.mark.skipif(not (O.RefLib.available("f32") and O.RefLib.available("f64")),
                                   reason="compiled reference (oracle/_ref) not built on this machine")


@ref_available
@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("seed", [3, 4])
def test_visibility_actors_vs_reference(prec, seed):
    o, r = O.Oracle(prec), O.RefLib(prec)
    w = synth.small_workload(seed=seed, grid_size=128, n_ant=14, n_time=6, num_planes=5, half_support=3,
                             oversampling=16)
    G, OS, us, ws = w.cfg.grid_size, 16, w.cfg.uv_scale, w.cfg.w_scale
    cfg = O.make_config(G, us, ws, OS)
    ov, ou, n = o.correct_to_finegrid(G, OS, w.uvw, w.vis, us)
    rv, ru, rn = r.correct_to_finegrid(cfg, G, OS, w.uvw, w.vis)
    np.testing.assert_array_equal(ou, ru)
    np.testing.assert_array_equal(
        o.std_gridding(G, OS, w.gkernels, w.supports, ou, w.vis, us, ws),
        r.std_gridding(cfg, G, OS, w.gkernels, w.supports, ou, w.vis))
    grid = np.random.default_rng(seed).standard_normal((G * G, 2))
    np.testing.assert_array_equal(o.std_degridding(G, OS, w.dkernels, w.supports, grid, ou, us, ws),
                                  r.std_degridding(cfg, G, OS, w.dkernels, w.supports, grid, ou))
    np.testing.assert_array_equal(o.gridding_cpu(G, 16, w.gkernels, w.supports, w.uvw, w.vis, us, ws),
                                  r.gridding_actor(cfg, G, w.gkernels, w.supports, w.uvw, w.vis))


@ref_available
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_taper_kill_line_vs_reference(prec):
    """G = 2560 > 2458: the reference zeroes rows/columns at |i - G/2| = 1229."""
    o, r = O.Oracle(prec), O.RefLib(prec)
    G = 2560
    img = np.random.default_rng(5).standard_normal(G * G)
    p = o.half_prolate(G)
    out = o.conv_correction(G, img, p)
    np.testing.assert_array_equal(out, r.conv_correction(O.make_config(G, 1, 1), G, img, r.half_prolate_ext(G)))
    assert np.all(out.reshape(G, G)[:, G // 2 + 1229] == 0) and np.all(out.reshape(G, G)[G // 2 - 1229, :] == 0)


@ref_available
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_hogbom_vs_reference_with_wrap(prec):
    """Peaks in the lower-right quadrant make the reference's mirrored PSF
    index wrap to the next row and, on the last row, read psf[G*G]."""
    o, r = O.Oracle(prec), O.RefLib(prec)
    G = 48
    rng = np.random.default_rng(9)
    yy, xx = np.mgrid[0:G, 0:G]
    psf = np.exp(-((xx - G // 2) ** 2 + (yy - G // 2) ** 2) / 6.0)
    psf = (psf / psf.max()).reshape(-1)
    res = 0.001 * rng.standard_normal(G * G)
    for (x0, y0, a) in ((40, 5, 1.0), (30, 10, 0.7), (5, 40, 0.5), (44, 2, 0.8)):
        res += a * np.roll(np.roll(psf.reshape(G, G), y0 - G // 2, 0), x0 - G // 2, 1).reshape(-1)
    cfg = O.make_config(G, 1, 1, psf_max_value=3.0, cell_size=2e-4)
    n1, s1, m1, _ = o.hogbom(G, 150, 200, res, psf, 3.0, 2e-4)
    n2, s2, m2 = r.hogbom(cfg, G, 150, 200, res, psf)
    assert n1 == n2
    np.testing.assert_array_equal(s1, s2)
    np.testing.assert_array_equal(m1, m2)


@ref_available
def test_prolate_vs_reference():
    o, r = O.Oracle("f64"), O.RefLib("f64")
    for nu in np.linspace(0, 1.2, 97):
        assert o.prolate_spheroidal(nu) == r.lib.prolate_spheroidal(O._d(nu))
