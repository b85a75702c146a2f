"""Every branch of the warp-per-visibility kernels against the oracle.

The kernels pick their path per plan and per batch of four visibilities:

* plans with a power-of-two oversampling get quad records (per-visibility
  quadrant bases into the degridding table and its conjugated copy) and
  batches of four half-support-4 fast visibilities run from them; other
  oversampling factors keep the geometry-record paths;
* the gridding half of the fused pass and the plain grid pass reuse the
  degridding samples when the two kernel sets are equal or conjugate (sign
  +1 / -1 on the imaginary part) and read the gridding set otherwise.

Each case runs the fused pass (convolutional degridding), the plain degrid
pass and the plain grid pass on one seeded workload of half support 4 and
compares them with the oracle (degridgrid.c:69-125, 147-191): predicted
visibilities and grids within GRID_TOL relative RMS, and grids touching
exactly the cells the oracle touches.
"""
from __future__ import annotations

import numpy as np
import pytest

import synth
from conftest import rel_rms

pytestmark = pytest.mark.gpu

GRID_TOL = 2e-6


def _touched(g):
    return np.abs(np.asarray(g)).sum(1) != 0


def _workload(os_):
    # 96 antennas in a disc, 24 time steps: 109,440 visibilities on a 256^2
    # grid, 6 w-planes of half support 4
    return synth.make_workload(f"paths_os{os_}", 96, 800.0, "disc", 24, 256, 5, 0.05, 1.0, 1e-3, 6, 4,
                               oversampling=os_, seed=11)


def _kernel_sets(w, relation):
    g = w.gkernels
    if relation == "conjugate":  # the workload's own pair: degridding = conj(gridding)
        return g, w.dkernels
    if relation == "equal":
        return g, g.copy()
    # unrelated: the degridding set is a perturbed copy (neither equal nor conjugate)
    rng = np.random.default_rng(3)
    return g, (w.dkernels * (1.0 + 0.01 * rng.standard_normal(w.dkernels.shape))).astype(np.float32)


@pytest.mark.parametrize("os_", [16, 12])
@pytest.mark.parametrize("relation", ["conjugate", "equal", "unrelated"])
def test_fast_kernel_paths_vs_oracle(sdp, device, oracle32, os_, relation):
    import torch
    w = _workload(os_)
    G, OS = w.cfg.grid_size, os_
    us, ws = w.cfg.uv_scale, w.cfg.w_scale
    gk_h, dk_h = _kernel_sets(w, relation)
    _, ou, _ = oracle32.correct_to_finegrid(G, OS, w.uvw, w.vis, us)
    dev = torch.device("cuda", 0)
    uvw = torch.from_numpy(ou).to(dev)
    gk = torch.from_numpy(gk_h).to(dev)
    dk = torch.from_numpy(dk_h).to(dev)
    sup = torch.from_numpy(w.supports).to(dev)
    rng = np.random.default_rng(5)
    model = (rng.standard_normal((G * G, 2)) * 1e-2).astype(np.float32)
    model_d = torch.from_numpy(model).to(dev)
    meas = torch.from_numpy(w.vis).to(dev)
    plan = device.plan(G, OS, us, ws, uvw, sdp.Device.wkernels(gk, sup, w.supports),
                       sdp.Device.wkernels(dk, sup, w.supports), keep=(uvw, gk, dk, sup))
    try:
        plan.set_measured(meas)
        res = torch.empty((G * G, 2), dtype=torch.float32, device=dev)
        pred = torch.empty_like(meas)
        plan.cycle(model_d, res, sdp.SDP_DEGRID_CONV, predicted=pred)
        pred2 = torch.empty_like(meas)
        plan.degrid(model_d, pred2, sdp.SDP_DEGRID_CONV)
        grid = torch.zeros((G * G, 2), dtype=torch.float32, device=dev)
        plan.grid(meas, grid)
        torch.cuda.synchronize()
        plan.check_flags()
    finally:
        plan.close()
    p_ref = oracle32.std_degridding(G, OS, dk_h, w.supports, model, ou, us, ws, nearest=False)
    r_ref = oracle32.std_gridding(G, OS, gk_h, w.supports, ou, oracle32.subtract_vis(w.vis, p_ref), us, ws)
    g_ref = oracle32.std_gridding(G, OS, gk_h, w.supports, ou, w.vis, us, ws)
    for name, got, ref in (("cycle predicted", pred, p_ref), ("degrid", pred2, p_ref), ("cycle residual", res, r_ref),
                           ("grid", grid, g_ref)):
        got = got.cpu().numpy()
        assert rel_rms(got, ref) <= GRID_TOL, (name, rel_rms(got, ref))
        if got.shape[0] == G * G:
            np.testing.assert_array_equal(_touched(got), _touched(ref), err_msg=name)
