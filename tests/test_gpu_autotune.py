"""Plan shapes and the autotuner (no counterpart in the reference: the
reference grids one visibility at a time).

Every plan shape (uv tile side, visibilities per work item, lanes per
visibility) bins the same visibilities into other work items; gridding,
degridding and the fused major-cycle pass must give the default plan's
results up to the order of the floating-point sums (the default plan is
itself checked against the oracle in test_gpu_actors / test_gpu_pipeline).
The autotuner must return a shape from its candidate set whose plan gives
those results too.
"""
from __future__ import annotations

import numpy as np
import pytest

import synth
from conftest import rel_rms

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(sdp, device):
    import torch
    w = synth.small_workload(seed=13, grid_size=256, n_ant=40, n_time=24, num_planes=5, half_support=3,
                             oversampling=16, n_src=8)
    G, OS = w.cfg.grid_size, w.cfg.oversampling
    dev = torch.device("cuda", 0)
    uvw_raw = torch.from_numpy(w.uvw).to(dev)
    uvw = torch.empty_like(uvw_raw)
    device.correct_to_finegrid(G, OS, w.cfg.uv_scale, uvw_raw, uvw)
    gk = torch.from_numpy(w.gkernels).to(dev)
    dk = torch.from_numpy(w.dkernels).to(dev)
    sup = torch.from_numpy(w.supports).to(dev)
    wg = sdp.Device.wkernels(gk, sup, w.supports)
    wd = sdp.Device.wkernels(dk, sup, w.supports)
    meas = torch.from_numpy(w.vis).to(dev)
    rng = np.random.default_rng(1)
    model = torch.from_numpy((rng.standard_normal((G * G, 2)) * 1e-2).astype(np.float32)).to(dev)
    return dict(w=w, G=G, OS=OS, uvw=uvw, wg=wg, wd=wd, keep=(uvw, gk, dk, sup), meas=meas, model=model)


def _run(sdp, device, st, options):
    import torch
    w, G = st["w"], st["G"]
    plan = device.plan(G, st["OS"], w.cfg.uv_scale, w.cfg.w_scale, st["uvw"], st["wg"], st["wd"], keep=st["keep"],
                       options=options)
    plan.set_measured(st["meas"])
    res = torch.empty((G * G, 2), dtype=torch.float32, device="cuda")
    pred = torch.empty_like(st["meas"])
    plan.cycle(st["model"], res, sdp.SDP_DEGRID_CONV, predicted=pred)
    grid = torch.empty_like(res)
    plan.grid(st["meas"], grid)
    deg = torch.empty_like(pred)
    plan.degrid(st["model"], deg)
    torch.cuda.synchronize()
    plan.check_flags()
    opts = plan.options()
    plan.close()
    return res.cpu().numpy(), pred.cpu().numpy(), grid.cpu().numpy(), deg.cpu().numpy(), opts


@pytest.mark.parametrize("tile,chunk,lanes,warps", [(16, 512, 0, 0), (64, 2048, 0, 0), (32, 1024, 16, 0),
                                                    (64, 64, 32, 0), (8, 4096, 0, 0), (24, 256, 0, 4),
                                                    (32, 1024, 8, 0), (16, 300, 0, 8)])
def test_plan_shapes_agree(sdp, device, setup, tile, chunk, lanes, warps):
    """Warp-per-visibility kernel (lanes 0) and the group kernels (8 / 16 /
    32 lanes) over tile sides and work-item sizes against the default plan."""
    ref = _run(sdp, device, setup, None)
    got = _run(sdp, device, setup, sdp.PlanOptions(tile, chunk, lanes, warps))
    assert (got[4].tile, got[4].chunk, got[4].lanes, got[4].warps) == (tile, chunk, lanes, warps)
    assert (ref[4].tile, ref[4].chunk, ref[4].warps) == (16, 512, 4)  # sdp_visplan_create's shape
    for a, b in zip(got[:4], ref[:4]):
        assert rel_rms(a, b) <= 1e-6


def test_bad_options_rejected(sdp, device, setup):
    import torch
    w, G = setup["w"], setup["G"]
    for o in (sdp.PlanOptions(20, 0, 0), sdp.PlanOptions(0, 10, 0), sdp.PlanOptions(0, 0, 12),
              sdp.PlanOptions(0, 0, 8 if setup["w"].half_support > 4 else 4), sdp.PlanOptions(0, 0, 0, 6)):
        with pytest.raises(sdp.SdpError):
            device.plan(G, setup["OS"], w.cfg.uv_scale, w.cfg.w_scale, setup["uvw"], setup["wg"], setup["wd"],
                        keep=setup["keep"], options=o)


def test_autotune_picks_a_valid_shape(sdp, device, setup):
    import torch
    w, G = setup["w"], setup["G"]
    scratch = torch.empty((G * G, 2), dtype=torch.float32, device="cuda")
    best, ms, cand = device.autotune(G, setup["OS"], w.cfg.uv_scale, w.cfg.w_scale, setup["uvw"], setup["wg"],
                                     setup["wd"], setup["meas"], setup["model"], scratch)
    assert cand >= 20 and ms > 0
    assert best.tile in (8, 16, 24, 32) and best.chunk in (256, 512, 1024) and best.lanes in (0, 8, 16)
    assert best.warps in (0, 4, 8)
    ref = _run(sdp, device, setup, None)
    got = _run(sdp, device, setup, best)
    for a, b in zip(got[:4], ref[:4]):
        assert rel_rms(a, b) <= 1e-6
