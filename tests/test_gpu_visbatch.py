"""Several channels' fused visibility passes in one launch (sdp_visbatch).

Three channels of different sizes (one with a different w-plane count) are
run through one batched launch; every channel's residual grid must equal the
one its own plan's sdp_visplan_cycle gives (the same arithmetic; only the
order of the float atomics differs) and the oracle's degrid -> subtract ->
grid within the grid tolerance.
"""
from __future__ import annotations

import numpy as np
import pytest

import synth
from conftest import rel_rms

pytestmark = pytest.mark.gpu

SAME_CODE_TOL = 1e-6    # batched vs single-plan launch: atomics order only
ORACLE_TOL = 2e-5       # vs the oracle's sequential sums (degrid normalisation + gridding)


def _channels():
    specs = [dict(seed=51, n_ant=24, n_time=20, num_planes=5), dict(seed=52, n_ant=30, n_time=12, num_planes=5),
             dict(seed=53, n_ant=16, n_time=30, num_planes=7)]
    out = []
    for sp in specs:
        w = synth.small_workload(seed=sp["seed"], grid_size=256, n_ant=sp["n_ant"], n_time=sp["n_time"],
                                 num_planes=sp["num_planes"], half_support=3, oversampling=16)
        out.append(w)
    return out


def test_batch_matches_single_plans_and_oracle(sdp, device, oracle32):
    import torch
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(9)
    plans, models, residuals, singles, keep = [], [], [], [], []
    for w in _channels():
        G = w.cfg.grid_size
        gk = torch.from_numpy(w.gkernels).to(dev)
        dk = torch.from_numpy(w.dkernels).to(dev)
        sup = torch.from_numpy(w.supports).to(dev)
        uvw = torch.from_numpy(w.uvw).to(dev)
        meas = torch.from_numpy(w.vis).to(dev)
        plan = device.plan(G, w.cfg.oversampling, w.cfg.uv_scale, w.cfg.w_scale, uvw,
                           sdp.Device.wkernels(gk, sup, w.supports), sdp.Device.wkernels(dk, sup, w.supports),
                           keep=(uvw, gk, dk, sup))
        plan.set_measured(meas)
        model = torch.from_numpy((rng.standard_normal((G * G, 2)) * 1e-2).astype(np.float32)).to(dev)
        single = torch.empty_like(model)
        plan.cycle(model, single, sdp.SDP_DEGRID_CONV)
        plans.append(plan)
        models.append(model)
        residuals.append(torch.full_like(model, 7.0))  # the batch must zero it
        singles.append(single)
        keep.append(meas)
    batch = device.batch(plans)
    assert batch.num_work_items() == sum(p.num_work_items() for p in plans)
    batch.set_grids(models, residuals)
    for _ in range(2):  # a second cycle gives the same grids
        batch.cycle(sdp.SDP_DEGRID_CONV)
        torch.cuda.synchronize()
        for c, w in enumerate(_channels()):
            got = residuals[c].cpu().numpy()
            assert rel_rms(got, singles[c].cpu().numpy()) <= SAME_CODE_TOL, c
            G = w.cfg.grid_size
            pred = oracle32.std_degridding(G, w.cfg.oversampling, w.dkernels, w.supports, models[c].cpu().numpy(),
                                           w.uvw, w.cfg.uv_scale, w.cfg.w_scale, nearest=False)
            delta = oracle32.subtract_vis(w.vis, pred)
            ref = oracle32.std_gridding(G, w.cfg.oversampling, w.gkernels, w.supports, w.uvw, delta,
                                        w.cfg.uv_scale, w.cfg.w_scale)
            assert rel_rms(got, ref) <= ORACLE_TOL, (c, rel_rms(got, ref))
    batch.close()
    for p in plans:
        p.close()


def test_batch_rejects_mixed_plans(sdp, device):
    import torch
    dev = torch.device("cuda", 0)
    w = synth.small_workload(seed=60, grid_size=64)
    gk = torch.from_numpy(w.gkernels).to(dev)
    sup = torch.from_numpy(w.supports).to(dev)
    uvw = torch.from_numpy(w.uvw).to(dev)
    wk = sdp.Device.wkernels(gk, sup, w.supports)
    a = device.plan(64, w.cfg.oversampling, w.cfg.uv_scale, w.cfg.w_scale, uvw, wk, wk, keep=(uvw, gk, sup))
    b = device.plan(64, w.cfg.oversampling, w.cfg.uv_scale, w.cfg.w_scale, uvw, wk, wk,
                    mode=sdp.SDP_GRID_STD | sdp.SDP_PLAN_COORD_F64, keep=(uvw, gk, sup))
    with pytest.raises(sdp.SdpError):
        device.batch([a, b])
    a.close()
    b.close()
