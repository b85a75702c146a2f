"""Generated inputs: W-projection kernel tables and the dirty PSF on the GPU.

* kernel tables against the numpy construction of the same kernels
  (synth.wproj_kernels: FFT of the zero-padded screen) within float rounding,
  with the supports/offsets of the reference's layout (top.c:246-251);
* the dirty PSF of a plan against the oracle's PSF (unit visibilities
  gridded, transformed, taper-corrected, normalised: oracle.dirty_psf)
  within the pipeline's image tolerance, with the same maximum.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle as O
import synth
from conftest import rel_rms

pytestmark = pytest.mark.gpu

_i, _d, _p = C.c_int, C.c_double, C.c_void_p


@pytest.mark.parametrize("planes,hs,OS,max_w,fov,M", [(5, [3, 3, 3, 3, 3], 16, 800.0, 0.02, 256),
                                                     (4, [2, 3, 4, 4], 8, 3000.0, 0.05, 128)])
def test_wkernels_match_numpy(sdp, device, planes, hs, OS, max_w, fov, M):
    import torch
    lib = sdp.load()
    dev = torch.device("cuda", 0)
    hs_arr = (C.c_int * planes)(*hs)
    total = C.c_int(0)
    assert lib.sdp_wkernels_generate_sizes(_i(planes), hs_arr, _i(OS), C.byref(total)) == 0
    lib.sdp_wkernels_generate_scratch_bytes.restype = C.c_size_t
    nscr = lib.sdp_wkernels_generate_scratch_bytes(_i(planes), hs_arr, _i(OS))
    gk = torch.empty((total.value, 2), dtype=torch.float32, device=dev)
    dk = torch.empty_like(gk)
    sup = np.zeros((planes, 2), np.int32)
    scr = torch.empty(nscr, dtype=torch.uint8, device=dev)
    st = lib.sdp_wkernels_generate(_i(planes), hs_arr, _i(OS), _d(max_w), _d(fov), _i(M), _p(gk.data_ptr()),
                                   _p(dk.data_ptr()), sup.ctypes.data_as(_p), _p(scr.data_ptr()), C.c_size_t(nscr),
                                   None)
    assert st == 0, lib.sdp_last_error()
    g_ref, d_ref, s_ref = synth.wproj_kernels(planes, hs, OS, max_w, fov, image_samples=M)
    np.testing.assert_array_equal(sup, s_ref)
    g = gk.cpu().numpy()
    d = dk.cpu().numpy()
    scale = np.abs(g_ref).max()
    np.testing.assert_allclose(g, g_ref, rtol=0, atol=2e-6 * scale)
    np.testing.assert_array_equal(d[:, 0], g[:, 0])
    np.testing.assert_array_equal(d[:, 1], -g[:, 1])


def test_psf_generate_matches_oracle(sdp, device, oracle32):
    import torch
    lib = sdp.load()
    dev = torch.device("cuda", 0)
    w = synth.small_workload(seed=71, grid_size=256, n_ant=24, n_time=20, num_planes=5, half_support=3,
                             oversampling=16)
    G, OS = w.cfg.grid_size, w.cfg.oversampling
    psf_ref, mx_ref = O.dirty_psf(oracle32, G, OS, w.uvw, w.gkernels, w.supports, w.cfg.uv_scale, w.cfg.w_scale)
    uvw_raw = torch.from_numpy(w.uvw).to(dev)
    uvw = torch.empty_like(uvw_raw)
    device.correct_to_finegrid(G, OS, w.cfg.uv_scale, uvw_raw, uvw)
    gk = torch.from_numpy(w.gkernels).to(dev)
    sup = torch.from_numpy(w.supports).to(dev)
    wk = sdp.Device.wkernels(gk, sup, w.supports)
    plan = device.plan(G, OS, w.cfg.uv_scale, w.cfg.w_scale, uvw, wk, wk, keep=(uvw, gk, sup))
    prol = torch.empty(G // 2 + 1, dtype=torch.float32, device=dev)
    device.prolate_table(G, prol)
    ones = torch.empty((w.num_vis, 2), dtype=torch.float32, device=dev)
    grid = torch.empty((G * G, 2), dtype=torch.float32, device=dev)
    work = torch.empty_like(grid)
    psf = torch.empty(G * G, dtype=torch.float32, device=dev)
    mx = torch.zeros(1, dtype=torch.float64, device=dev)
    st = lib.sdp_psf_generate(plan.handle, _p(prol.data_ptr()), _p(ones.data_ptr()), _p(grid.data_ptr()),
                              _p(work.data_ptr()), _p(psf.data_ptr()), _p(mx.data_ptr()), None)
    assert st == 0, lib.sdp_last_error()
    torch.cuda.synchronize()
    got = psf.cpu().numpy()
    assert abs(float(mx.item()) - mx_ref) <= 1e-5 * abs(mx_ref)
    # compared in the gridded domain (times the taper), as the pipeline images are
    p = np.zeros(G // 2 + 1)
    p[: G // 2] = synth.prolate(np.arange(G // 2) / (G // 2))
    dd = np.abs(np.arange(G) - G // 2)
    t = np.outer(p[dd], p[dd]).reshape(-1)
    assert rel_rms(got * t, np.asarray(psf_ref, np.float64) * t) <= 2e-5
    assert got.max() == np.float32(1.0)
    plan.close()


def test_image_rms_fp64(sdp, device):
    import torch
    rng = np.random.default_rng(3)
    G = 300
    img = (rng.standard_normal(G * G) * 10.0 ** rng.integers(-3, 3, G * G)).astype(np.float32)
    got = device.image_rms(G, torch.from_numpy(img).cuda())
    ref = float(np.sqrt(np.mean(img.astype(np.float64) ** 2)))
    assert abs(got - ref) <= 1e-12 * ref
