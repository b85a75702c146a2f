"""The device-resident major cycle (sdp_pipeline) against the oracle's FFT
pipeline in the generated schedule's order (oracle.fft_pipeline).

* float-build coordinates (the reference's default PRECISION) against the
  float oracle: residual images within PIPE_TOL_F32 rel-RMS every cycle and
  the same components (positions exact, fluxes within FLUX_TOL of the
  brightest);
* FP64 coordinates (SDP_COORD_F64) against the FP64 oracle (the reference
  built at double PRECISION): every image within 1e-4 rel-RMS, the
  north-star bound;
* the CUDA-graph replay of the cycle against direct launches.

Images are compared after weighting by the taper the pipeline divides by
(convolution_correction_run.c:4-35), i.e. in the domain the FFT and the
gridding produce.  The taper goes to zero at the image edge, so next to the
edge the corrected image is rounding noise multiplied by up to 1e8; there
two runs of the same GPU code (or the float and double builds of the
reference) differ at 1e-4 and more, and an unweighted rel-RMS measures that
amplification, not the arithmetic.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
import synth
from conftest import rel_rms

pytestmark = pytest.mark.gpu

PIPE_TOL_F32 = 2e-5
FLUX_TOL = 5e-4
FP64_IMAGE_TOL = 1e-4


def _taper(G):
    p = np.zeros(G // 2 + 1)
    p[: G // 2] = synth.prolate(np.arange(G // 2) / (G // 2))
    d = np.abs(np.arange(G) - G // 2)
    return np.outer(p[d], p[d]).reshape(-1)


def weighted_rel_rms(a, b, G):
    t = _taper(G)
    return rel_rms(np.asarray(a, np.float64) * t, np.asarray(b, np.float64) * t)


def inner_rel_rms(a, b, G):
    """Unweighted rel-RMS over the inner half of the image (|x|, |y| < G/4
    from the centre), where the taper correction divides by at least
    prolate(1/2)^2 ~ 0.13."""
    sl = slice(G // 4, 3 * G // 4)
    a = np.asarray(a, np.float64).reshape(G, G)[sl, sl]
    b = np.asarray(b, np.float64).reshape(G, G)[sl, sl]
    return rel_rms(a, b)


def _setup(seed=17, G=256, minor=60):
    w = synth.small_workload(seed=seed, grid_size=G, n_ant=24, n_time=20, num_planes=5, half_support=3,
                             oversampling=16, n_src=6)
    n = w.num_vis - w.num_vis % 4
    uvw, vis = w.uvw[:n].copy(), w.vis[:n].copy()
    return w, uvw, vis, minor


def _gpu_pipeline(sdp, device, w, uvw, vis, psf, psf_max, cycles, minor, coord, nearest, graph):
    import torch
    dev = torch.device("cuda", 0)
    G = w.cfg.grid_size
    gk = torch.from_numpy(w.gkernels).to(dev)
    dk = torch.from_numpy(w.dkernels).to(dev)
    sup = torch.from_numpy(w.supports).to(dev)
    cfg = sdp.PipelineConfig(G, 16, w.cfg.uv_scale, w.cfg.w_scale, w.cfg.cell_size, minor, 200, 0.1, 1.5, 0.0002,
                             psf_max, sdp.SDP_DEGRID_NEAREST if nearest else sdp.SDP_DEGRID_CONV, coord, 1,
                             1 if graph else 0)
    uvw_d = torch.from_numpy(uvw).to(dev)
    vis_d = torch.from_numpy(vis).to(dev)
    psf_d = torch.from_numpy(np.ascontiguousarray(psf, dtype=np.float32)).to(dev)
    pl = device.pipeline(cfg, uvw_d, vis_d, psf_d, sdp.Device.wkernels(gk, sup, w.supports),
                         sdp.Device.wkernels(dk, sup, w.supports), keep=(gk, dk, sup))
    outs = []
    for _ in range(cycles):
        pl.major_cycle()
        outs.append(pl.outputs())
    graph_on = pl.graph_active()
    if graph and not graph_on:
        print("graph capture refused:", pl.graph_error())
    pl.close()
    return outs, graph_on


@pytest.mark.parametrize("nearest", [True, False])
def test_pipeline_float_build_matches_oracle(sdp, device, oracle32, nearest):
    w, uvw, vis, minor = _setup()
    G = w.cfg.grid_size
    psf, psf_max = O.dirty_psf(oracle32, G, 16, uvw, w.gkernels, w.supports, w.cfg.uv_scale, w.cfg.w_scale)
    ref = O.fft_pipeline(oracle32, G, 16, uvw, vis, w.gkernels, w.dkernels, w.supports, w.cfg.uv_scale,
                         w.cfg.w_scale, psf, psf_max, w.cfg.cell_size, 3, minor, 200, nearest=nearest)
    got, _ = _gpu_pipeline(sdp, device, w, uvw, vis, psf, psf_max, 3, minor, sdp.SDP_COORD_F32, nearest, False)
    for k, ((img_r, model_r, n_r, src_r), (img_g, model_g, src_g, n_g)) in enumerate(zip(ref, got)):
        assert weighted_rel_rms(img_g, img_r, G) <= PIPE_TOL_F32, (k, weighted_rel_rms(img_g, img_r, G))
        assert n_g == n_r
        np.testing.assert_array_equal(src_g[:, :2], src_r[:, :2])
        # fluxes within FLUX_TOL of the brightest component: a component's flux
        # is loop_gain x the residual at its pixel, and a single pixel carries
        # up to ~10x the image's rel-RMS rounding (atomics and FFT order)
        np.testing.assert_allclose(src_g[:, 2], src_r[:, 2], rtol=0, atol=FLUX_TOL * np.abs(src_r[:, 2]).max())
        assert rel_rms(model_g, model_r) <= 1e-4


def test_pipeline_fp64_coordinates_within_1e4_of_fp64_oracle(sdp, device, oracle64, record_property):
    """Every image within 1e-4 rel-RMS of the FP64 oracle, taper-weighted
    (the domain the FFT and gridding produce); the unweighted figures over
    the inner half and over the whole image (dominated by the edge pixels,
    where the taper correction divides by ~1e-8) are recorded beside it."""
    w, uvw, vis, minor = _setup(seed=23)
    G = w.cfg.grid_size
    psf, psf_max = O.dirty_psf(oracle64, G, 16, uvw, w.gkernels, w.supports, w.cfg.uv_scale, w.cfg.w_scale)
    ref = O.fft_pipeline(oracle64, G, 16, uvw, vis, w.gkernels, w.dkernels, w.supports, w.cfg.uv_scale,
                         w.cfg.w_scale, psf, psf_max, w.cfg.cell_size, 3, minor, 200, nearest=False)
    got, _ = _gpu_pipeline(sdp, device, w, uvw, vis, psf.astype(np.float32), psf_max, 3, minor,
                           sdp.SDP_COORD_F64, False, False)
    for k, ((img_r, model_r, n_r, src_r), (img_g, model_g, src_g, n_g)) in enumerate(zip(ref, got)):
        wr, ir, ur = weighted_rel_rms(img_g, img_r, G), inner_rel_rms(img_g, img_r, G), rel_rms(img_g, img_r)
        record_property(f"cycle{k}_rel_rms", {"taper_weighted": wr, "unweighted_inner_half": ir,
                                               "unweighted_whole_image": ur})
        assert wr <= FP64_IMAGE_TOL, (k, wr)
        assert n_g == n_r
        np.testing.assert_array_equal(src_g[:, :2], src_r[:, :2].astype(np.float32))


def test_visplan_fp64_coordinates_match_fp64_build(sdp, device, golden):
    """Edge-of-grid and within-one-ulp points: SDP_COORD_F64 selects the taps
    the reference's double build selects (grid_f64 fixture)."""
    import torch
    d = golden("wproj_g64.npz")
    dev = torch.device("cuda", 0)
    G, OS = int(d["grid_size"]), int(d["oversampling"])
    gk = torch.from_numpy(d["gkernels"]).to(dev)
    sup = torch.from_numpy(d["supports"]).to(dev)
    wk = sdp.Device.wkernels(gk, sup, d["supports"])
    uvw = torch.from_numpy(d["uvw"]).to(dev)
    vis = torch.from_numpy(d["vis"]).to(dev)
    grid = torch.empty((G * G, 2), dtype=torch.float32, device=dev)
    plan = device.plan(G, OS, float(d["uv_scale"]), float(d["w_scale"]), uvw, wk, wk,
                       mode=sdp.SDP_GRID_STD | sdp.SDP_PLAN_COORD_F64 | sdp.SDP_PLAN_SNAP, keep=(uvw, gk, sup))
    plan.grid(vis, grid)
    torch.cuda.synchronize()
    out = grid.cpu().numpy()
    ref = d["grid_f64"]
    assert rel_rms(out, ref) <= 2e-6
    np.testing.assert_array_equal(np.abs(out).sum(1) == 0, np.abs(ref).sum(1) == 0)
    plan.close()


def test_pipeline_graph_replay_matches_direct(sdp, device, oracle32):
    w, uvw, vis, minor = _setup(seed=29, G=128, minor=30)
    G = w.cfg.grid_size
    psf, psf_max = O.dirty_psf(oracle32, G, 16, uvw, w.gkernels, w.supports, w.cfg.uv_scale, w.cfg.w_scale)
    direct, _ = _gpu_pipeline(sdp, device, w, uvw, vis, psf, psf_max, 3, minor, sdp.SDP_COORD_F32, True, False)
    graph, graph_on = _gpu_pipeline(sdp, device, w, uvw, vis, psf, psf_max, 3, minor, sdp.SDP_COORD_F32, True, True)
    for (img_a, model_a, src_a, n_a), (img_b, model_b, src_b, n_b) in zip(direct, graph):
        assert weighted_rel_rms(img_b, img_a, G) <= 1e-5
        assert n_a == n_b
    assert graph_on, "graph capture refused"


@pytest.mark.parametrize("nearest", [True, False])
def test_pipeline_c1_configuration(sdp, device, oracle32, nearest):
    """The reference's own CPU configuration at full size: 64 antennas in a
    2 km disc, 60 time steps (120,960 visibilities, 50 sources plus 1 mJy
    noise), 512^2, 8 w-planes of support 7, OS 16, 3 major cycles of 200
    Hogbom minor cycles.  Residual images within PIPE_TOL_F32 x (cycle + 1)
    (differences compound through the model), component positions exact and
    fluxes within FLUX_TOL up to the first near-tie pick; later cycles compare
    residual levels."""
    w = synth.workload_c1(seed=1, compute_vis=True)
    n = w.num_vis - w.num_vis % 4
    uvw, vis = w.uvw[:n].copy(), w.vis[:n].copy()
    G = w.cfg.grid_size
    psf, psf_max = O.dirty_psf(oracle32, G, 16, uvw, w.gkernels, w.supports, w.cfg.uv_scale, w.cfg.w_scale)
    ref = O.fft_pipeline(oracle32, G, 16, uvw, vis, w.gkernels, w.dkernels, w.supports, w.cfg.uv_scale,
                         w.cfg.w_scale, psf, psf_max, w.cfg.cell_size, 3, 200, 200, nearest=nearest)
    got, graph_on = _gpu_pipeline(sdp, device, w, uvw, vis, psf, psf_max, 3, 200, sdp.SDP_COORD_F32, nearest, True)
    assert graph_on
    diverged = False
    t = _taper(G)
    for k, ((img_r, model_r, n_r, src_r), (img_g, model_g, src_g, n_g)) in enumerate(zip(ref, got)):
        if not diverged:
            # rounding differences reach the next cycle through the model, so the
            # bound grows with the cycle (cycle 0: PIPE_TOL_F32)
            tol = PIPE_TOL_F32 * (1 + k)
            assert weighted_rel_rms(img_g, img_r, G) <= tol, (k, weighted_rel_rms(img_g, img_r, G))
            assert n_g == n_r, (k, n_g, n_r)
            diverged = not _components_agree(src_g[:n_g], src_r[:n_r], k)
        else:
            # after a tie was broken the other way, each run continues from its
            # own (equally valid) model: their residual levels must still agree
            rms_g = np.sqrt(np.mean((np.asarray(img_g, np.float64) * t) ** 2))
            rms_r = np.sqrt(np.mean((np.asarray(img_r, np.float64) * t) ** 2))
            assert abs(rms_g - rms_r) <= 1e-3 * rms_r, (k, rms_g, rms_r)


def _components_agree(src_g, src_r, cycle):
    """Component lists agree up to a near-tie.  Hogbom takes the first pixel
    of largest |r|; with 200 minor cycles on a 50-source sky some pick two
    pixels whose |r| differ by less than the images' rounding, and either is
    the reference's choice.  Positions must be identical up to the first
    such pick; there the two lists' fluxes must be equal within FLUX_TOL of
    the brightest (a tie, not an error), and from there on each list is a
    valid Hogbom continuation, so only the images are compared."""
    scale = np.abs(src_r[:, 2]).max()
    diff = np.flatnonzero(np.any(src_g[:, :2] != src_r[:, :2], axis=1))
    d = int(diff[0]) if diff.size else len(src_r)
    np.testing.assert_allclose(src_g[:d, 2], src_r[:d, 2], rtol=0, atol=FLUX_TOL * scale)
    if d < len(src_r):
        assert abs(abs(src_g[d, 2]) - abs(src_r[d, 2])) <= FLUX_TOL * scale, (cycle, d, src_g[d], src_r[d])
    return d == len(src_r)
