"""Parity of the fused visibility pass at the sizes the benchmark runs.

The smaller parity tests (test_gpu_actors, test_gpu_pipeline) pin the index
arithmetic on toy grids; these run the device path on the workloads whose
throughput is reported, with the plan shape the autotuner picks there:

* the 256-antenna, 10 km spiral channel: 3,916,800 visibilities, 2048^2,
  17 w-planes of half support 4, OS 16 (the single-channel workload);
* one channel of the 512-antenna, 40 km spiral at 8192^2 with 64 w-planes
  (kernels generated on the GPU), a seeded subset of 1.2 M visibilities
  through the full-size plan;
* four channels of the 64-channel, 100-200 MHz batch (real per-channel
  visibility counts after their seeded 0-60 % flags, 32 w-planes) in one
  batched launch.

Checks (tolerances stated here):
* convolutional mode (degridgrid.c:147-191 without the nearest-cell
  override) against the oracle restatement: predicted visibilities and the
  residual grid within GRID_TOL rel-RMS, and the residual grid touches
  exactly the cells the oracle touches;
* nearest-cell mode (the reference's std_degridding as shipped,
  degridgrid.c:193-200) against the reference's own actors compiled from its
  sources (oracle/_ref): predicted visibilities bit-exact, residual grid
  within GRID_TOL with the identical touched-cell pattern.

The oracle runs on all host threads: the visibilities are cut into slices
(ctypes releases the GIL), each slice grids into its own grid, and the grids
are summed in float64.  Only the summation order differs from a one-thread
run; the comparison tolerance covers that.
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import channels
import oracle as O
import synth
from conftest import rel_rms

pytestmark = pytest.mark.gpu

GRID_TOL = 2e-6


def _threads(limit=32):
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    return max(1, min(limit, n))


def oracle_cycle(o, G, OS, gk, dk, sup, uvw, meas, model, us, ws, nearest, threads):
    """degrid (oracle) -> measured - predicted -> grid (oracle), sliced over
    host threads; returns (predicted, residual grid in float64)."""
    n = uvw.shape[0]
    cuts = np.linspace(0, n, threads + 1).astype(np.int64)

    def run(k):
        a, b = cuts[k], cuts[k + 1]
        u = np.ascontiguousarray(uvw[a:b])
        p = o.std_degridding(G, OS, dk, sup, model, u, us, ws, nearest=nearest)
        d = o.subtract_vis(np.ascontiguousarray(meas[a:b]), p)
        return p, o.std_gridding(G, OS, gk, sup, u, d, us, ws)

    with ThreadPoolExecutor(max_workers=threads) as ex:
        parts = list(ex.map(run, range(threads)))
    pred = np.concatenate([p for p, _ in parts], axis=0)
    grid = np.zeros((G * G, 2), np.float64)
    for _, g in parts:
        grid += g
    return pred, grid


def ref_cycle_nearest(lib, cfg, G, OS, gk, dk, sup, uvw, meas, model, threads):
    """The same pass through the reference's compiled actors (nearest-cell
    std_degridding as shipped, subtract_from_measurements_finegrid,
    std_gridding)."""
    n = uvw.shape[0]
    cuts = np.linspace(0, n, threads + 1).astype(np.int64)

    def run(k):
        a, b = cuts[k], cuts[k + 1]
        u = np.ascontiguousarray(uvw[a:b])
        p = lib.std_degridding(cfg, G, OS, dk, sup, model, u)
        d = lib.subtract_finegrid(np.ascontiguousarray(meas[a:b]), p)
        return p, lib.std_gridding(cfg, G, OS, gk, sup, u, d)

    with ThreadPoolExecutor(max_workers=threads) as ex:
        parts = list(ex.map(run, range(threads)))
    pred = np.concatenate([p for p, _ in parts], axis=0)
    grid = np.zeros((G * G, 2), np.float64)
    for _, g in parts:
        grid += g
    return pred, grid


def touched(g):
    return np.abs(np.asarray(g)).sum(1) != 0


def _device_inputs(sdp, device, w, G, OS, uvw_host, gk_h, dk_h, sup_h, seed):
    import torch
    dev = torch.device("cuda", 0)
    uvw_raw = torch.from_numpy(uvw_host).to(dev)
    uvw = torch.empty_like(uvw_raw)
    device.correct_to_finegrid(G, OS, w.cfg.uv_scale, uvw_raw, uvw)
    gk = torch.from_numpy(gk_h).to(dev)
    dk = torch.from_numpy(dk_h).to(dev)
    sup = torch.from_numpy(sup_h).to(dev)
    rng = np.random.default_rng(seed)
    model = (rng.standard_normal((G * G, 2)) * 1e-3).astype(np.float32)
    return dict(uvw=uvw, gk=gk, dk=dk, sup=sup, wg=sdp.Device.wkernels(gk, sup, sup_h),
                wd=sdp.Device.wkernels(dk, sup, sup_h), model=model, model_d=torch.from_numpy(model).to(dev))


def _device_cycle(sdp, device, w, G, OS, d, meas_h, options, mode):
    import torch
    meas = torch.from_numpy(meas_h).to("cuda")
    plan = device.plan(G, OS, w.cfg.uv_scale, w.cfg.w_scale, d["uvw"], d["wg"], d["wd"],
                       keep=(d["uvw"], d["gk"], d["dk"], d["sup"]), options=options)
    plan.set_measured(meas)
    res = torch.empty((G * G, 2), dtype=torch.float32, device="cuda")
    pred = torch.empty_like(meas)
    plan.cycle(d["model_d"], res, mode, predicted=pred)
    torch.cuda.synchronize()
    plan.check_flags()
    opts = plan.options()
    plan.close()
    return pred.cpu().numpy(), res.cpu().numpy(), opts


@pytest.fixture(scope="module")
def c2(sdp, device):
    import torch
    w = synth.make_workload("c2_2048", 256, 5000.0, "spiral", 120, 2048, 200, 1e-3, 1.0, 1e-4, 17, 4,
                            freq_hz=140e6, seed=2, compute_vis=False)
    G, OS = w.cfg.grid_size, w.cfg.oversampling
    d = _device_inputs(sdp, device, w, G, OS, w.uvw, w.gkernels, w.dkernels, w.supports, seed=31)
    meas = torch.from_numpy(w.vis).to("cuda")
    res = torch.empty((G * G, 2), dtype=torch.float32, device="cuda")
    shape, _, _ = device.autotune(G, OS, w.cfg.uv_scale, w.cfg.w_scale, d["uvw"], d["wg"], d["wd"], meas,
                                  d["model_d"], res, reps=2)
    d["shape"] = shape
    d["uvw_h"] = d["uvw"].cpu().numpy()
    return w, G, OS, d


def test_c2_fused_pass_conv_autotuned_shape_vs_oracle(sdp, device, c2, oracle32):
    w, G, OS, d = c2
    assert w.num_vis == 3_916_800
    pred, res, opts = _device_cycle(sdp, device, w, G, OS, d, w.vis, d["shape"], sdp.SDP_DEGRID_CONV)
    assert (opts.tile, opts.chunk, opts.lanes) == (d["shape"].tile, d["shape"].chunk, d["shape"].lanes)
    p_ref, g_ref = oracle_cycle(oracle32, G, OS, w.gkernels, w.dkernels, w.supports, d["uvw_h"], w.vis, d["model"],
                                w.cfg.uv_scale, w.cfg.w_scale, nearest=False, threads=_threads())
    assert rel_rms(pred, p_ref) <= GRID_TOL, rel_rms(pred, p_ref)
    assert rel_rms(res, g_ref) <= GRID_TOL, rel_rms(res, g_ref)
    np.testing.assert_array_equal(touched(res), touched(g_ref))


def test_c2_fused_pass_nearest_vs_compiled_reference(sdp, device, c2):
    if not O.RefLib.available("f32"):
        pytest.skip("the compiled reference (oracle/_ref) is not built")
    w, G, OS, d = c2
    pred, res, _ = _device_cycle(sdp, device, w, G, OS, d, w.vis, d["shape"], sdp.SDP_DEGRID_NEAREST)
    lib = O.RefLib("f32")
    cfg = O.make_config(G, w.cfg.uv_scale, w.cfg.w_scale, OS)
    p_ref, g_ref = ref_cycle_nearest(lib, cfg, G, OS, w.gkernels, w.dkernels, w.supports, d["uvw_h"], w.vis,
                                     d["model"], threads=_threads())
    np.testing.assert_array_equal(pred, p_ref)
    assert rel_rms(res, g_ref) <= GRID_TOL, rel_rms(res, g_ref)
    np.testing.assert_array_equal(touched(res), touched(g_ref))


def test_c2_every_candidate_shape_vs_oracle(sdp, device, c2, oracle32):
    """Every tile side / work-item size the autotuner may choose, on the full
    workload, against one oracle pass."""
    w, G, OS, d = c2
    p_ref, g_ref = oracle_cycle(oracle32, G, OS, w.gkernels, w.dkernels, w.supports, d["uvw_h"], w.vis, d["model"],
                                w.cfg.uv_scale, w.cfg.w_scale, nearest=False, threads=_threads())
    t_ref = touched(g_ref)
    for tile in (16, 32, 64):
        for chunk in (512, 2048):
            pred, res, _ = _device_cycle(sdp, device, w, G, OS, d, w.vis, sdp.PlanOptions(tile, chunk, 0),
                                         sdp.SDP_DEGRID_CONV)
            assert rel_rms(pred, p_ref) <= GRID_TOL, (tile, chunk, rel_rms(pred, p_ref))
            assert rel_rms(res, g_ref) <= GRID_TOL, (tile, chunk, rel_rms(res, g_ref))
            np.testing.assert_array_equal(touched(res), t_ref)


def test_c5_channel_8192_subset_vs_oracle(sdp, device, oracle32):
    """8192^2, 64 generated w-planes of half support 4: a seeded 1.2 M subset
    of the 40 km channel through the full-size plan (autotuned shape)."""
    import torch
    w = synth.make_workload("c5_8192", 512, 20000.0, "spiral", 200, 8192, 1, 1e-3, 1.0, 1e-4, 64, 4,
                            freq_hz=140e6, seed=5, compute_vis=False)
    G, OS = w.cfg.grid_size, w.cfg.oversampling
    rng = np.random.default_rng(55)
    sel = np.sort(rng.choice(w.num_vis, 1_200_000, replace=False))
    uvw_h = np.ascontiguousarray(w.uvw[sel])
    meas_h = np.ascontiguousarray(w.vis[sel])
    fov = w.cfg.cell_size * G
    gk, dk, sup = device.wkernels_generate([4] * 64, OS, w.cfg.max_w, fov)
    gk_h, dk_h, sup_h = gk.cpu().numpy(), dk.cpu().numpy(), sup.cpu().numpy()
    d = _device_inputs(sdp, device, w, G, OS, uvw_h, gk_h, dk_h, sup_h, seed=57)
    meas = torch.from_numpy(meas_h).to("cuda")
    res = torch.empty((G * G, 2), dtype=torch.float32, device="cuda")
    shape, _, _ = device.autotune(G, OS, w.cfg.uv_scale, w.cfg.w_scale, d["uvw"], d["wg"], d["wd"], meas,
                                  d["model_d"], res, reps=1)
    del res
    pred, res, _ = _device_cycle(sdp, device, w, G, OS, d, meas_h, shape, sdp.SDP_DEGRID_CONV)
    uvw_s = d["uvw"].cpu().numpy()
    p_ref, g_ref = oracle_cycle(oracle32, G, OS, gk_h, dk_h, sup_h, uvw_s, meas_h, d["model"], w.cfg.uv_scale,
                                w.cfg.w_scale, nearest=False, threads=_threads(8))
    assert rel_rms(pred, p_ref) <= GRID_TOL, rel_rms(pred, p_ref)
    assert rel_rms(res, g_ref) <= GRID_TOL, rel_rms(res, g_ref)
    np.testing.assert_array_equal(touched(res), touched(g_ref))


def test_c3_batch_four_channels_vs_oracle(sdp, device, oracle32):
    """Four channels of the 64-channel batch (100-200 MHz, per-channel flags
    0-60 %, 32 w-planes hs 4) at their real visibility counts, one batched
    launch, each channel's residual grid against the oracle."""
    import torch
    nch, f_lo, f_hi = 64, 100e6, 200e6
    base = synth.make_workload("c3_base", 256, 5000.0, "spiral", 120, 2048, 1, 1e-3, 1.0, 1e-4, 32, 4,
                               freq_hz=f_hi, seed=3, compute_vis=False)
    G, OS = base.cfg.grid_size, base.cfg.oversampling
    counts = channels.flagged_counts(nch, base.num_vis, seed=11)
    pick = (0, 21, 42, 63)
    dev = torch.device("cuda", 0)
    gk = torch.from_numpy(base.gkernels).to(dev)
    dk = torch.from_numpy(base.dkernels).to(dev)
    sup = torch.from_numpy(base.supports).to(dev)
    wg = sdp.Device.wkernels(gk, sup, base.supports)
    wd = sdp.Device.wkernels(dk, sup, base.supports)
    rng = np.random.default_rng(77)
    model = (rng.standard_normal((G * G, 2)) * 1e-3).astype(np.float32)
    model_d = torch.from_numpy(model).to(dev)
    plans, resid, hosts = [], [], []
    for c in pick:
        f = f_lo + (f_hi - f_lo) * c / (nch - 1)
        sel = np.sort(np.random.default_rng(1000 + c).choice(base.num_vis, counts[c], replace=False))
        uvw_h = np.ascontiguousarray(base.uvw[sel] * np.float32(f / f_hi))
        meas_h = (0.1 * np.random.default_rng(2000 + c).standard_normal((counts[c], 2))).astype(np.float32)
        uvw_raw = torch.from_numpy(uvw_h).to(dev)
        uvw = torch.empty_like(uvw_raw)
        device.correct_to_finegrid(G, OS, base.cfg.uv_scale, uvw_raw, uvw)
        pl = device.plan(G, OS, base.cfg.uv_scale, base.cfg.w_scale, uvw, wg, wd, keep=(uvw, gk, dk, sup))
        pl.set_measured(torch.from_numpy(meas_h).to(dev))
        plans.append(pl)
        resid.append(torch.empty((G * G, 2), dtype=torch.float32, device=dev))
        hosts.append((uvw.cpu().numpy(), meas_h))
    assert min(counts[c] for c in pick) >= 1_500_000
    batch = device.batch(plans)
    batch.set_grids([model_d] * len(pick), resid)
    batch.cycle(sdp.SDP_DEGRID_CONV)
    torch.cuda.synchronize()
    for pl in plans:
        pl.check_flags()
    for k, (uvw_h, meas_h) in enumerate(hosts):
        _, g_ref = oracle_cycle(oracle32, G, OS, base.gkernels, base.dkernels, base.supports, uvw_h, meas_h, model,
                                base.cfg.uv_scale, base.cfg.w_scale, nearest=False, threads=_threads())
        got = resid[k].cpu().numpy()
        assert rel_rms(got, g_ref) <= GRID_TOL, (pick[k], rel_rms(got, g_ref))
        np.testing.assert_array_equal(touched(got), touched(g_ref))
    batch.close()
    for pl in plans:
        pl.close()
