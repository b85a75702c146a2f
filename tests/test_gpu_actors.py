"""GPU parity of every actor drop-in, called through the exported C symbols
of libsdp_b200.so with host buffers, against the oracle and the golden
fixtures of the compiled reference.

Tolerances (stated here, checked below):
* index work (nearest-cell degridding, fine-grid snap, shifts, taper,
  subtraction, merge, prolate table): bit-exact with the float reference;
* gridding / g2g: same taps and kernel samples as the float reference; only
  the order of the float additions differs (shared-memory subgrids and
  atomic flushes), so grids agree to rel-RMS <= GRID_TOL;
* FFT: rel-RMS <= FFT_TOL against the FP64 oracle transform;
* DFT: rel-RMS <= DFT_TOL against the FP64 oracle (FP64 phase on the GPU);
* Hogbom on an identical residual: components and model bit-exact.
"""
from __future__ import annotations

import numpy as np
import pytest

import synth
from conftest import rel_rms

pytestmark = pytest.mark.gpu

GRID_TOL = 2e-6
FFT_TOL = 2e-6
DFT_TOL = 2e-6


def cfg_for(sdp, d):
    return sdp.make_config(int(d["grid_size"]), float(d["uv_scale"]), float(d["w_scale"]), int(d["oversampling"]))


def test_correct_to_finegrid_bit_exact(sdp, actors, golden):
    d = golden("wproj_g64.npz")
    cfg = cfg_for(sdp, d)
    ov, ou, n = actors.correct_to_finegrid(cfg, int(d["grid_size"]), int(d["oversampling"]), d["uvw"], d["vis"])
    assert n == d["uvw"].shape[0]
    np.testing.assert_array_equal(ou, d["ctf_uvw_f32"])
    np.testing.assert_array_equal(ov, d["ctf_vis_f32"])


def test_std_gridding_matches_reference(sdp, actors, golden):
    d = golden("wproj_g64.npz")
    cfg = cfg_for(sdp, d)
    G, OS = int(d["grid_size"]), int(d["oversampling"])
    for uvw_key, ref_key in (("ctf_uvw_f32", "grid_f32"), ("uvw", "grid_raw_f32")):
        g = actors.std_gridding(cfg, G, OS, d["gkernels"], d["supports"], d[uvw_key], d["vis"])
        assert rel_rms(g, d[ref_key]) <= GRID_TOL
        # every cell the reference touched is touched, and no other
        np.testing.assert_array_equal(np.abs(g).sum(1) == 0, np.abs(d[ref_key]).sum(1) == 0)


def test_std_gridding_vs_oracle_random(sdp, actors, oracle32, oracle64):
    w = synth.small_workload(seed=21, grid_size=128, n_ant=20, n_time=10, num_planes=5, half_support=3,
                             oversampling=16)
    G, OS = w.cfg.grid_size, 16
    cfg = sdp.make_config(G, w.cfg.uv_scale, w.cfg.w_scale, OS)
    _, ou, _ = oracle32.correct_to_finegrid(G, OS, w.uvw, w.vis, w.cfg.uv_scale)
    g = actors.std_gridding(cfg, G, OS, w.gkernels, w.supports, ou, w.vis)
    ref32 = oracle32.std_gridding(G, OS, w.gkernels, w.supports, ou, w.vis, w.cfg.uv_scale, w.cfg.w_scale)
    assert rel_rms(g, ref32) <= GRID_TOL


def test_std_degridding_nearest_bit_exact(sdp, actors, golden):
    d = golden("wproj_g64.npz")
    cfg = cfg_for(sdp, d)
    G, OS = int(d["grid_size"]), int(d["oversampling"])
    actors.set_degrid_mode(sdp.SDP_DEGRID_NEAREST)
    out = actors.std_degridding(cfg, G, OS, d["dkernels"], d["supports"], d["model_grid"], d["ctf_uvw_f32"])
    np.testing.assert_array_equal(out, d["degrid_f32"])
    out = actors.std_degridding(cfg, G, OS, d["dkernels"], d["supports"], d["model_grid"], d["uvw"])
    np.testing.assert_array_equal(out, d["degrid_raw_f32"])


def test_std_degridding_conv_vs_oracle(sdp, actors, oracle32, golden):
    d = golden("wproj_g64.npz")
    cfg = cfg_for(sdp, d)
    G, OS = int(d["grid_size"]), int(d["oversampling"])
    us, ws = float(d["uv_scale"]), float(d["w_scale"])
    actors.set_degrid_mode(sdp.SDP_DEGRID_CONV)
    try:
        out = actors.std_degridding(cfg, G, OS, d["dkernels"], d["supports"], d["model_grid"], d["ctf_uvw_f32"])
    finally:
        actors.set_degrid_mode(sdp.SDP_DEGRID_NEAREST)
    ref = oracle32.std_degridding(G, OS, d["dkernels"], d["supports"], d["model_grid"], d["ctf_uvw_f32"], us, ws,
                                  nearest=False)
    assert rel_rms(out, ref) <= GRID_TOL


def test_degrid_tail_entries_zeroed(sdp, actors, golden):
    """Only *num_corrected_visibilities entries are computed; the rest of the
    NUM_VISIBILITIES output is zero (degridgrid.c:132)."""
    d = golden("wproj_g64.npz")
    cfg = cfg_for(sdp, d)
    G, OS = int(d["grid_size"]), int(d["oversampling"])
    out = np.full((d["uvw"].shape[0], 2), 7.0, dtype=np.float32)
    actors.std_degridding(cfg, G, OS, d["dkernels"], d["supports"], d["model_grid"], d["ctf_uvw_f32"], num=100,
                          out=out)
    np.testing.assert_array_equal(out[:100], d["degrid_f32"][:100])
    assert np.all(out[100:] == 0)


def test_subtract_from_measurements_bit_exact(actors, golden):
    d = golden("wproj_g64.npz")
    np.testing.assert_array_equal(actors.subtract_finegrid(d["vis"], d["degrid_f32"]), d["subtract_f32"])


def test_g2g_degridgrid_matches_reference(sdp, actors, golden):
    d = golden("wproj_g64.npz")
    cfg = cfg_for(sdp, d)
    G, OS = int(d["grid_size"]), int(d["oversampling"])
    out = actors.g2g_degridgrid(cfg, G, OS, d["gkernels"], d["supports"], d["dkernels"], d["supports"],
                                d["model_grid"], d["ctf_uvw_f32"])
    assert rel_rms(out, d["g2g_f32"]) <= GRID_TOL


def test_gridding_actor_matches_reference(sdp, actors, golden):
    d = golden("wproj_g64.npz")
    cfg = cfg_for(sdp, d)
    g = actors.gridding_actor(cfg, int(d["grid_size"]), d["gkernels"], d["supports"], d["uvw"], d["vis"])
    assert rel_rms(g, d["gridding_actor_f32"]) <= GRID_TOL


def test_gridding_cpu_accumulates(sdp, actors, oracle32, golden):
    d = golden("wproj_g64.npz")
    G = int(d["grid_size"])
    start = np.random.default_rng(1).standard_normal((G * G, 2)).astype(np.float32)
    g = actors.gridding_cpu(start, d["gkernels"], d["supports"], d["uvw"], d["vis"], 16, G, float(d["uv_scale"]),
                            float(d["w_scale"]))
    ref = oracle32.gridding_cpu(G, 16, d["gkernels"], d["supports"], d["uvw"], d["vis"], float(d["uv_scale"]),
                                float(d["w_scale"]), grid=start)
    assert rel_rms(g, ref) <= GRID_TOL


def test_shifts_bit_exact(sdp, actors, golden):
    d = golden("fft_g32.npz")
    G = int(d["grid_size"])
    cfg = sdp.make_config(G, 1.0, 1.0)
    np.testing.assert_array_equal(actors.fft_shift_c2c(cfg, G, d["x"]), d["shift_c2c_f32"])
    np.testing.assert_array_equal(actors.fft_shift_c2r(cfg, G, d["x"]), d["shift_c2r_f32"])
    np.testing.assert_array_equal(actors.fft_shift_r2c(cfg, G, d["image"]), d["shift_r2c_f32"])


@pytest.mark.parametrize("G", [16, 32, 64, 128, 512, 1024, 2048])
def test_fft_vs_fp64_oracle(actors, oracle64, G):
    x = np.random.default_rng(G).standard_normal((G * G, 2)).astype(np.float32)
    for inverse in (False, True):
        out = actors.fft(G, x, inverse)
        ref = oracle64.fft2d(G, x, +1 if inverse else -1)
        assert rel_rms(out, ref) <= FFT_TOL, (G, inverse)


def test_fft_golden(actors, golden):
    d = golden("fft_g32.npz")
    G = int(d["grid_size"])
    assert rel_rms(actors.fft(G, d["x"], False), d["fft_fwd_f64"]) <= FFT_TOL
    assert rel_rms(actors.fft(G, d["x"], True), d["fft_inv_f64"]) <= FFT_TOL


def test_prolate_and_taper_bit_exact(sdp, actors, golden):
    d = golden("fft_g32.npz")
    G = int(d["grid_size"])
    cfg = sdp.make_config(G, 1.0, 1.0)
    p = actors.half_prolate(G)
    np.testing.assert_array_equal(p, d["prolate_f32"][: G // 2])
    np.testing.assert_array_equal(actors.conv_correction(cfg, G, d["image"], p), d["taper_f32"])


@pytest.mark.parametrize("G", [512, 2048, 2560])
def test_prolate_table_and_kill_line(sdp, actors, oracle32, G):
    p = actors.half_prolate(G)
    ref = oracle32.half_prolate(G)
    np.testing.assert_array_equal(p, ref[: G // 2])
    img = np.random.default_rng(G).standard_normal(G * G).astype(np.float32)
    np.testing.assert_array_equal(actors.conv_correction(sdp.make_config(G, 1, 1), G, img, p),
                                  oracle32.conv_correction(G, img, ref))


def test_merge_and_image_subtract_bit_exact(actors, golden):
    d = golden("fft_g32.npz")
    G = int(d["grid_size"])
    np.testing.assert_array_equal(actors.merge_grids(G, d["grids4"]), d["merge_f32"])
    np.testing.assert_array_equal(actors.subtract_image(G, d["image"], d["image"][::-1].copy()), d["subimg_f32"])


def test_add_visibilities(actors):
    rng = np.random.default_rng(0)
    a = rng.standard_normal((1000, 2)).astype(np.float32)
    b = rng.standard_normal((1000, 2)).astype(np.float32)
    np.testing.assert_array_equal(actors.add_visibilities(a, b), a + b)


def test_dft_vs_fp64_oracle(sdp, actors, oracle32, golden):
    d = golden("dft.npz")
    cfg = sdp.make_config(64, 1.0, 1.0)
    out = actors.dft(cfg, d["sources"], d["uvw"])
    assert rel_rms(out, d["vis_f64"]) <= DFT_TOL
    # the float reference's own error against FP64 is larger than the GPU's
    assert rel_rms(out, d["vis_f64"]) <= rel_rms(d["vis_f32"], d["vis_f64"]) + 1e-7


def test_dft_long_baselines(sdp, actors, oracle64):
    """|u l| up to ~1e3 cycles: the FP64 phase keeps the error at FP32 level."""
    rng = np.random.default_rng(4)
    uvw = rng.uniform(-4.0e4, 4.0e4, size=(2000, 3)).astype(np.float32)
    src = np.stack([rng.uniform(-0.03, 0.03, 50), rng.uniform(-0.03, 0.03, 50), rng.uniform(0.01, 1, 50)], 1)
    src = src.astype(np.float32)
    out = actors.dft(sdp.make_config(64, 1.0, 1.0), src, uvw)
    assert rel_rms(out, oracle64.dft(src, uvw)) <= 1e-5


def test_hogbom_bit_exact(sdp, actors, golden):
    d = golden("hogbom_g64.npz")
    G = int(d["grid_size"])
    cfg = sdp.make_config(G, 1.0, 1.0, psf_max_value=float(d["psf_max"]), cell_size=float(d["cell_size"]))
    n, src, model = actors.hogbom(cfg, G, 100, 200, d["dirty"], d["psf"])
    assert n == int(d["num_sources"])
    np.testing.assert_array_equal(src, d["sources"])
    np.testing.assert_array_equal(model, d["model"])


def test_hogbom_wrap_and_cap(sdp, actors, oracle32):
    """Peaks that make the mirrored PSF index wrap (and read psf[G*G]); more
    minor cycles than MAX_SOURCES stores only the first MAX_SOURCES."""
    G = 48
    rng = np.random.default_rng(9)
    yy, xx = np.mgrid[0:G, 0:G]
    psf = np.exp(-((xx - G // 2) ** 2 + (yy - G // 2) ** 2) / 6.0)
    psf = (psf / psf.max()).reshape(-1).astype(np.float32)
    res = (0.001 * rng.standard_normal(G * G)).astype(np.float32)
    for (x0, y0, a) in ((40, 5, 1.0), (30, 10, 0.7), (5, 40, 0.5), (44, 2, 0.8)):
        res += (a * np.roll(np.roll(psf.reshape(G, G), y0 - G // 2, 0), x0 - G // 2, 1)).reshape(-1).astype(np.float32)
    cfg = sdp.make_config(G, 1.0, 1.0, psf_max_value=3.0, cell_size=2e-4)
    n1, s1, m1, _ = oracle32.hogbom(G, 150, 200, res, psf, 3.0, 2e-4)
    n2, s2, m2 = actors.hogbom(cfg, G, 150, 200, res, psf)
    assert n1 == n2
    np.testing.assert_array_equal(s1, s2)
    np.testing.assert_array_equal(m1, m2)
    n3, s3, m3 = actors.hogbom(cfg, G, 150, 40, res, psf)
    assert n3 == 40
    np.testing.assert_array_equal(s3, s1[:40])
    np.testing.assert_array_equal(m3, m1)


def test_clean_psf_matches_reference(sdp, actors, golden):
    d = golden("hogbom_g64.npz")
    G = int(d["grid_size"])
    cfg = sdp.make_config(G, 1.0, 1.0, psf_max_value=float(d["psf_max"]))
    clean, hd = actors.clean_psf(cfg, G, d["psf"])
    np.testing.assert_array_equal(hd, d["halfdims"])
    assert rel_rms(clean, d["clean_psf"]) <= 1e-6


def test_empty_and_error_paths(sdp, actors, golden):
    d = golden("wproj_g64.npz")
    cfg = cfg_for(sdp, d)
    G, OS = int(d["grid_size"]), int(d["oversampling"])
    g = actors.std_gridding(cfg, G, OS, d["gkernels"], d["supports"], d["uvw"][:0], d["vis"][:0])
    assert not np.any(g)
    with pytest.raises(sdp.SdpError) as e:
        actors.correct_to_finegrid(cfg, G, OS, d["uvw"], d["vis"], simplify=1)
    assert e.value.status == 1
    # a w beyond the kernel tables is reported, not read out of bounds
    bad = d["uvw"].copy()
    bad[0, 2] = 1e9
    with pytest.raises(sdp.SdpError) as e:
        actors.std_gridding(cfg, G, OS, d["gkernels"], d["supports"], bad, d["vis"])
    assert e.value.status == 6
    with pytest.raises(sdp.SdpError):
        actors.fft(24, np.zeros((24 * 24, 2), np.float32), False)


@pytest.mark.parametrize("G", [1024, 2048])
def test_hogbom_large_bit_exact_vs_oracle(sdp, actors, oracle32, G):
    """The persistent on-chip CLEAN (G <= ~2750) against the oracle at full size."""
    rng = np.random.default_rng(G)
    yy, xx = np.mgrid[0:G, 0:G]
    psf = np.exp(-((xx - G // 2) ** 2 + (yy - G // 2) ** 2) / 18.0).astype(np.float32)
    psf /= psf.max()
    res = (0.001 * rng.standard_normal((G, G))).astype(np.float32)
    for _ in range(40):
        x0, y0 = rng.integers(8, G - 8, 2)
        res += (rng.uniform(0.05, 1.0) * np.roll(np.roll(psf, y0 - G // 2, 0), x0 - G // 2, 1)).astype(np.float32)
    res, psf = res.reshape(-1), psf.reshape(-1)
    cfg = sdp.make_config(G, 1.0, 1.0, psf_max_value=4.0, cell_size=1e-5)
    n1, s1, m1, _ = oracle32.hogbom(G, 200, 200, res, psf, 4.0, 1e-5)
    n2, s2, m2 = actors.hogbom(cfg, G, 200, 200, res, psf)
    assert n1 == n2 == 200
    np.testing.assert_array_equal(s2, s1)
    np.testing.assert_array_equal(m2, m1)


@pytest.mark.parametrize("G,psf_offset", [(1024, 0), (2048, 0), (2048, 1), (1500, 0), (1001, 0)])
def test_hogbom_persistent_sidelobes_vs_oracle(sdp, device, oracle32, G, psf_offset):
    """Persistent CLEAN through the device entry point against the oracle,
    with a PSF whose sidelobes are nonzero everywhere (so every PSF sample of
    the window, the x-mirrored rows, the wrap into the next PSF row and the
    reads past the PSF's end all enter the residual), peaks up to the image
    edges: components, model and the final residual bit for bit.
    psf_offset = 1 passes a PSF that starts 4 bytes into its allocation.
    Pass variants: four pixels per thread and step (1024, 2048, 2048 with
    the offset PSF, 1500), one pixel per step (1001)."""
    import torch
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(G + 7 * psf_offset)
    yy, xx = np.mgrid[0:G, 0:G]
    psf = np.exp(-((xx - G // 2) ** 2 + (yy - G // 2) ** 2) / 8.0) + 2e-3 * rng.standard_normal((G, G))
    psf = (psf / psf.max()).astype(np.float32)
    res = 0.01 * rng.standard_normal((G, G))
    for _ in range(30):
        x0, y0 = rng.integers(0, G, 2)
        res += rng.uniform(0.1, 1.0) * np.roll(np.roll(psf, y0 - G // 2, 0), x0 - G // 2, 1)
    res, psf = res.astype(np.float32).reshape(-1), psf.reshape(-1)
    minor = 120
    n1, s1, m1, r1 = oracle32.hogbom(G, minor, minor, res, psf, 1.0, 1e-5)
    params = sdp.CleanParams(G, minor, minor, 0.1, 1.5, 0.0002, 1.0, 1e-5)
    pbuf = torch.zeros(G * G + 4, dtype=torch.float32, device=dev)
    pbuf[psf_offset:psf_offset + G * G] = torch.from_numpy(psf).to(dev)
    psf_d = pbuf[psf_offset:psf_offset + G * G]
    r = torch.from_numpy(res.copy()).to(dev)
    m = torch.zeros(G * G, dtype=torch.float32, device=dev)
    s = torch.zeros((minor, 3), dtype=torch.float32, device=dev)
    c = torch.zeros(1, dtype=torch.int32, device=dev)
    ws = torch.empty(device.hogbom_workspace_bytes(G), dtype=torch.uint8, device=dev)
    device.hogbom(params, r, psf_d, m, s, c, ws)
    torch.cuda.synchronize()
    n2 = int(c.item())
    assert n1 == n2 > 20
    np.testing.assert_array_equal(s[:n2].cpu().numpy(), s1)
    np.testing.assert_array_equal(m.cpu().numpy(), m1)
    np.testing.assert_array_equal(r.cpu().numpy(), r1)


@pytest.mark.parametrize("G", [1024, 1500])
def test_hogbom_noise_stop_vs_oracle(sdp, device, oracle32, G):
    """noise_factor x gain above 1, so the noise test (|max| < noise x mean
    |r| x gain, deconvolution_run.c:238) can end the loop: a few sources on
    noise, cleaned until only noise is left.  The persistent kernel then
    carries the sum of |r| through every minor cycle; the stop, components,
    model and residual must match the oracle."""
    import torch
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(G + 3)
    yy, xx = np.mgrid[0:G, 0:G]
    psf = np.exp(-((xx - G // 2) ** 2 + (yy - G // 2) ** 2) / 8.0)
    psf = (psf / psf.max()).astype(np.float32)
    res = 0.01 * rng.standard_normal((G, G))
    for _ in range(6):
        x0, y0 = rng.integers(G // 4, 3 * G // 4, 2)
        res += rng.uniform(0.5, 1.0) * np.roll(np.roll(psf, y0 - G // 2, 0), x0 - G // 2, 1)
    res, psf = res.astype(np.float32).reshape(-1), psf.reshape(-1)
    minor, gain, noise = 400, 0.1, 80.0
    n1, s1, m1, r1 = oracle32.hogbom(G, minor, minor, res, psf, 1.0, 1e-5, loop_gain=gain, noise_factor=noise)
    params = sdp.CleanParams(G, minor, minor, gain, noise, 0.0002, 1.0, 1e-5)
    r = torch.from_numpy(res.copy()).to(dev)
    psf_d = torch.from_numpy(psf).to(dev)
    m = torch.zeros(G * G, dtype=torch.float32, device=dev)
    s = torch.zeros((minor, 3), dtype=torch.float32, device=dev)
    c = torch.zeros(1, dtype=torch.int32, device=dev)
    ws = torch.empty(device.hogbom_workspace_bytes(G), dtype=torch.uint8, device=dev)
    device.hogbom(params, r, psf_d, m, s, c, ws)
    torch.cuda.synchronize()
    n2 = int(c.item())
    assert 10 < n1 < minor, n1  # the noise test ended the loop
    assert n2 == n1
    np.testing.assert_array_equal(s[:n2].cpu().numpy(), s1)
    np.testing.assert_array_equal(m.cpu().numpy(), m1)
    np.testing.assert_array_equal(r.cpu().numpy(), r1)


def test_hogbom_general_path_vs_oracle(sdp, device, oracle32):
    """G = 2816: the image no longer fits in shared memory over all SMs, so
    CLEAN runs as one launch per minor cycle (the general path, also the
    pipeline's fallback when a capture of the cooperative launch is refused);
    components, model and final residual bit for bit against the oracle,
    with a PSF whose sidelobes are nonzero everywhere."""
    import torch
    dev = torch.device("cuda", 0)
    G, minor = 2816, 60
    rng = np.random.default_rng(G)
    yy, xx = np.mgrid[0:G, 0:G]
    psf = np.exp(-((xx - G // 2) ** 2 + (yy - G // 2) ** 2) / 8.0) + 2e-3 * rng.standard_normal((G, G))
    psf = (psf / psf.max()).astype(np.float32)
    res = 0.01 * rng.standard_normal((G, G))
    for _ in range(20):
        x0, y0 = rng.integers(0, G, 2)
        res += rng.uniform(0.1, 1.0) * np.roll(np.roll(psf, y0 - G // 2, 0), x0 - G // 2, 1)
    res, psf = res.astype(np.float32).reshape(-1), psf.reshape(-1)
    n1, s1, m1, r1 = oracle32.hogbom(G, minor, minor, res, psf, 1.0, 1e-5)
    params = sdp.CleanParams(G, minor, minor, 0.1, 1.5, 0.0002, 1.0, 1e-5)
    r = torch.from_numpy(res.copy()).to(dev)
    m = torch.zeros(G * G, dtype=torch.float32, device=dev)
    s = torch.zeros((minor, 3), dtype=torch.float32, device=dev)
    c = torch.zeros(1, dtype=torch.int32, device=dev)
    ws = torch.empty(device.hogbom_workspace_bytes(G), dtype=torch.uint8, device=dev)
    device.hogbom(params, r, torch.from_numpy(psf).to(dev), m, s, c, ws)
    torch.cuda.synchronize()
    n2 = int(c.item())
    assert n1 == n2 > 20
    np.testing.assert_array_equal(s[:n2].cpu().numpy(), s1)
    np.testing.assert_array_equal(m.cpu().numpy(), m1)
    np.testing.assert_array_equal(r.cpu().numpy(), r1)


def test_bounded_wait_reports_timeout(sdp):
    """Failure detection without a GPU fault: a grid barrier that one arrival
    short of complete gives up after its bounded wait and reports
    SDP_ERR_TIMEOUT; the context stays usable afterwards."""
    import ctypes as C
    import torch
    lib = sdp.load()
    st = C.c_int(-1)
    sdp.check(lib.sdp_selftest_bounded_wait(C.c_int(4), C.c_longlong(200_000), C.byref(st)), lib)
    assert st.value == 5  # SDP_ERR_TIMEOUT
    x = torch.ones(1024, device="cuda")
    assert float(x.sum().item()) == 1024.0
