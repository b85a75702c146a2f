"""Benchmark: visibilities gridded + degridded per second on B200.

One step = one major-cycle visibility pass of the FFT imaging pipeline over
every visibility of the workload: W-projection degridding of the model grid
(convolutional, the value degridgrid.c:147-191 computes), subtraction from
the measured visibilities (gains_apply_run.c:273-297) and W-projection
gridding of the residual visibilities (degridgrid.c:69-125).  Workload: the
256-antenna, 10 km log-spiral array, 120 time steps -> 3,916,800
visibilities, 2048^2 grid, 17 w-planes of half support 4, oversampling 16
(seeded synthetic data; no public dataset is used).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

value: device-resident throughput (inputs in HBM, L2 flushed between timed
steps, CUDA events, max over ranks).  e2e: the same pass through the
reference-facing C ABI (std_degridding, subtract_from_measurements_finegrid,
std_gridding) with pinned host buffers and the host<->device copies inside
the timed region.  --impl reference times the reference's own actor code
compiled from its sources (oracle/_ref) on the host cores.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG = ROOT / "simsdp-generic-imaging-pipeline_b200"
sys.path.insert(0, str(PKG))

import channels  # noqa: E402
import synth  # noqa: E402

METRIC = "vis/s gridded+degridded"
UNIT = "vis/s"
PROFILES = ROOT / "profiles"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-major-cycle", action="store_true")
    ap.add_argument("--no-c3", action="store_true", help="skip the batched 64-channel pass")
    ap.add_argument("--no-c5", action="store_true", help="skip the 8192^2 single-channel measurement")
    ap.add_argument("--no-c4", action="store_true", help="skip the learned-proposal comparison")
    ap.add_argument("--c4-skies", type=int, default=16, help="held-out skies of the learned-proposal comparison")
    ap.add_argument("--cpu-sample", type=int, default=200_000, help="visibilities per CPU-baseline step")
    return ap.parse_args()


def workload(rank: int):
    """C2-shaped workload; each rank images its own frequency channel (weak
    scaling by channel, the reference's spectral parallelism)."""
    freq = 140e6 * (1.0 + 0.05 * rank)
    return synth.make_workload("c2_2048", 256, 5000.0, "spiral", 120, 2048, 200, 1e-3, 1.0, 1e-4, 17, 4,
                               freq_hz=freq, seed=2 + rank, compute_vis=False)


def algorithmic_bytes(n_vis: int, G: int) -> int:
    """Compulsory HBM bytes of one fused pass: uvw (12 B) and measured vis (8 B)
    read once per visibility, model grid read and residual grid written once."""
    return n_vis * (12 + 8) + 2 * 8 * G * G


def algorithmic_flops(n_vis: int, taps: int) -> int:
    """Complex multiply-add per tap in both directions: 8 flops x 2."""
    return n_vis * taps * 16


def read_profile_value(kernel: str, key: str):
    """A per-launch figure ("key: value") from the committed ncu summary."""
    f = PROFILES / f"{kernel}.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith(key + ":"):
            try:
                return int(float(line.split(":", 1)[1].split()[0]))
            except ValueError:
                return None
    return None


def read_traffic(kernel: str):
    """dram bytes per launch from the committed ncu summary, if present."""
    return read_profile_value(kernel, "traffic_bytes_per_launch")


class ClockSampler:
    """SM clock and clock-event (throttle) reasons, read through NVML every
    ~2 ms in a background thread; mark() opens and closes the window whose
    samples are summarised (the timed region).  Reading only."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.window = [None, None]
        self._stop = threading.Event()
        self.thread = None
        self.ok = False

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
            self.thread = threading.Thread(target=self._run, daemon=True)
            self.thread.start()
        except Exception:
            self.ok = False
        return self

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                try:
                    reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                except AttributeError:
                    reasons = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                self.samples.append((time.perf_counter(), mhz, reasons))
            except Exception:
                pass
            time.sleep(0.002)

    def mark(self, which: int):
        self.window[which] = time.perf_counter()

    def __exit__(self, *exc):
        self._stop.set()
        if self.thread:
            self.thread.join(timeout=2)

    def summary(self):
        if not self.ok:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "source": "nvml unavailable"}
        t0, t1 = self.window
        sel = [s for s in self.samples if (t0 is None or s[0] >= t0) and (t1 is None or s[0] <= t1)]
        if not sel:
            sel = self.samples[-5:]
        reasons = set()
        for _, _, r in sel:
            for name, bit in self.REASONS.items():
                if r & bit:
                    reasons.add(name)
        return {"sm_mhz": statistics.median([s[1] for s in sel]) if sel else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "samples": len(sel), "source": "nvml, 2 ms"}


# ---------------------------------------------------------------------------
# Reference arm / CPU baseline: the reference's actors on the host cores
# ---------------------------------------------------------------------------
def cpu_reference_pass(w, uvw_c, model_grid, sample: int, threads: int):
    """Runs std_degridding + subtract_from_measurements_finegrid + std_gridding
    of the reference (compiled from its sources, oracle/_ref; the oracle port
    when that is absent) on `sample` visibilities split over `threads` slices,
    as the reference's SLICES schedule does, and returns (seconds, kind)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    G, OS = w.cfg.grid_size, w.cfg.oversampling
    cfg = O.make_config(G, w.cfg.uv_scale, w.cfg.w_scale, OS)
    if O.RefLib.available("f32", "fast"):
        lib, kind = O.RefLib("f32", "fast"), "reference"
    elif O.RefLib.available("f32"):
        lib, kind = O.RefLib("f32"), "reference"
    else:
        lib, kind = None, "port"
    o = O.Oracle("f32") if lib is None else None
    idx = np.linspace(0, uvw_c.shape[0] - 1, sample).astype(np.int64)
    uvw = np.ascontiguousarray(uvw_c[idx])
    vis = np.ascontiguousarray(w.vis[idx])
    slices = np.array_split(np.arange(sample), threads)

    def run(sl):
        u = np.ascontiguousarray(uvw[sl])
        v = np.ascontiguousarray(vis[sl])
        if lib is not None:
            pred = lib.std_degridding(cfg, G, OS, w.dkernels, w.supports, model_grid, u)
            delta = lib.subtract_finegrid(v, pred)
            return lib.std_gridding(cfg, G, OS, w.gkernels, w.supports, u, delta)
        pred = o.std_degridding(G, OS, w.dkernels, w.supports, model_grid, u, w.cfg.uv_scale, w.cfg.w_scale, False)
        delta = o.subtract_vis(v, pred)
        return o.std_gridding(G, OS, w.gkernels, w.supports, u, delta, w.cfg.uv_scale, w.cfg.w_scale)

    # silence the reference's progress printf
    devnull = os.open(os.devnull, os.O_WRONLY)
    saved = os.dup(1)
    sys.stdout.flush()
    os.dup2(devnull, 1)
    try:
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=threads) as ex:
            grids = list(ex.map(run, slices))
        if lib is not None and len(grids) > 1:
            lib.merge_grids(G, np.concatenate(grids, axis=0))
        t1 = time.perf_counter()
    finally:
        sys.stdout.flush()
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)
    return t1 - t0, kind


def cpu_threads() -> int:
    """Host threads for the CPU arm: every core, up to 64 (each slice owns a
    full G^2 grid, as in the reference's SLICES schedule)."""
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    return max(1, min(64, n))


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    w = workload(0)
    G = w.cfg.grid_size
    threads = cpu_threads()
    rng = np.random.default_rng(5)
    model_grid = (rng.standard_normal((G * G, 2)) * 1e-3).astype(np.float32)
    uvw_c = snap_host(w)
    sample = max(threads * 2000, args.cpu_sample)
    for _ in range(max(0, args.warmup)):
        cpu_reference_pass(w, uvw_c, model_grid, min(sample, 20_000), threads)
    times = []
    kind = "port"
    for _ in range(args.steps):
        t, kind = cpu_reference_pass(w, uvw_c, model_grid, sample, threads)
        times.append(t)
    t = statistics.mean(times)
    value = sample / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{w.name}: {w.num_vis} vis, G=2048, 17 w-planes hs=4 OS=16; "
                               f"bounded sample of {sample} vis per step", "degrid": "convolutional"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{sample} visibilities of the workload per step, {threads} slices"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def snap_host(w):
    """Fine-grid snap of the uvw (degridgrid.c:24-25, 52-54), on the host in
    numpy with the reference's rounding; used only to feed the CPU arm the
    same coordinates the GPU arm grids."""
    G, OS, us = w.cfg.grid_size, w.cfg.oversampling, w.cfg.uv_scale
    u = w.uvw.astype(np.float64)
    fx = np.trunc((u[:, 0] * us + G // 2) * OS + 0.5)
    fy = np.trunc((u[:, 1] * us + G // 2) * OS + 0.5)
    out = np.empty_like(w.uvw)
    out[:, 0] = ((fx / OS - G // 2) / us).astype(np.float32)
    out[:, 1] = ((fy / OS - G // 2) / us).astype(np.float32)
    out[:, 2] = w.uvw[:, 2]
    return out


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def c3_block(S, D, dev, reps: int = 5):
    """The batched multi-channel workload: the 256-antenna layout at 64
    channels over 100-200 MHz, seeded per-channel flag fractions of 0-60 %
    (uneven visibility counts), 32 w-planes of half support 4, OS 16, one
    2048^2 grid per channel.  All channels' fused passes run in one
    persistent launch (sdp_visbatch); the same passes as 64 separate plan
    launches are timed beside it.  Inputs resident in HBM (4+ GB, larger than
    L2)."""
    import torch

    nch, f_lo, f_hi = 64, 100e6, 200e6
    base = synth.make_workload("c3_base", 256, 5000.0, "spiral", 120, 2048, 1, 1e-3, 1.0, 1e-4, 32, 4,
                               freq_hz=f_hi, seed=3, compute_vis=False)
    G, OS = base.cfg.grid_size, base.cfg.oversampling
    n_full = base.num_vis
    counts = channels.flagged_counts(nch, n_full, seed=11)
    gk = torch.from_numpy(base.gkernels).to(dev)
    dk = torch.from_numpy(base.dkernels).to(dev)
    sup = torch.from_numpy(base.supports).to(dev)
    wk_g = S.Device.wkernels(gk, sup, base.supports)
    wk_d = S.Device.wkernels(dk, sup, base.supports)
    uvw_top = torch.from_numpy(base.uvw).to(dev)
    plans, resid, keep = [], [], []
    gen = torch.Generator(device=dev)
    for c in range(nch):
        f = f_lo + (f_hi - f_lo) * c / (nch - 1)
        gen.manual_seed(1000 + c)
        sel = torch.randperm(n_full, device=dev, generator=gen)[:counts[c]].sort().values
        uvw = (uvw_top[sel] * (f / f_hi)).contiguous()
        meas = 0.1 * torch.randn((counts[c], 2), device=dev, generator=gen)
        pl = D.plan(G, OS, base.cfg.uv_scale, base.cfg.w_scale, uvw, wk_g, wk_d, keep=(uvw, gk, dk, sup))
        pl.set_measured(meas)
        plans.append(pl)
        resid.append(torch.empty((G * G, 2), dtype=torch.float32, device=dev))
        keep.append(meas)
    del uvw_top
    model = (1e-3 * torch.randn((G * G, 2), device=dev, generator=gen)).contiguous()
    batch = D.batch(plans)
    batch.set_grids([model] * nch, resid)

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return statistics.median(ts)

    def separate():
        for pl, r in zip(plans, resid):
            pl.cycle(model, r, S.SDP_DEGRID_CONV)

    t_batch = timed(lambda: batch.cycle(S.SDP_DEGRID_CONV))
    t_sep = timed(separate)
    total = int(sum(counts))
    out = {"workload": "64 channels 100-200 MHz, 256 antennas 10 km spiral, 120 time steps, per-channel flags "
                       "0-60 %, G=2048 per channel, 32 w-planes hs=4 OS=16",
           "vis_total": total, "vis_min": int(min(counts)), "vis_max": int(max(counts)),
           "work_items": batch.num_work_items(),
           "ms_batched": t_batch, "vis_per_s_batched": total / (t_batch * 1e-3),
           "ms_64_launches": t_sep, "vis_per_s_64_launches": total / (t_sep * 1e-3)}
    batch.close()
    for pl in plans:
        pl.close()
    del resid, keep, model
    torch.cuda.empty_cache()
    return out


def c5_block(S, D, dev, reps: int = 3):
    """One channel of the large g2g-scale workload: 512 antennas on a seeded
    40 km log spiral, 200 time steps (26,163,200 visibilities), 8192^2 grid,
    64 w-planes of half support 4 (kernels generated on the GPU), OS 16.
    Times the plan build, the fused visibility pass and a whole major cycle
    (graph; 200 Hogbom minor cycles on 8192^2, the one-launch-per-cycle
    path)."""
    import torch

    w = synth.make_workload("c5_8192", 512, 20000.0, "spiral", 200, 8192, 1, 1e-3, 1.0, 1e-4, 64, 4,
                            freq_hz=140e6, seed=5, compute_vis=False)
    G, OS, N = w.cfg.grid_size, w.cfg.oversampling, w.num_vis
    fov = w.cfg.cell_size * G
    gk, dk, sup = D.wkernels_generate([4] * 64, OS, w.cfg.max_w, fov)
    sup_h = sup.cpu().numpy()
    wk_g = S.Device.wkernels(gk, sup, sup_h)
    wk_d = S.Device.wkernels(dk, sup, sup_h)
    uvw_raw = torch.from_numpy(w.uvw).to(dev)
    uvw = torch.empty_like(uvw_raw)
    D.correct_to_finegrid(G, OS, w.cfg.uv_scale, uvw_raw, uvw)
    del uvw_raw
    gen = torch.Generator(device=dev).manual_seed(23)
    meas = 0.1 * torch.randn((N, 2), device=dev, generator=gen)

    def ev_time(fn, n):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(n):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return statistics.median(ts)

    plans = []
    t_plan = ev_time(lambda: plans.append(D.plan(G, OS, w.cfg.uv_scale, w.cfg.w_scale, uvw, wk_g, wk_d,
                                                 keep=(uvw, gk, dk, sup))), 2)
    for pl in plans[:-1]:
        pl.close()
    plan = plans[-1]
    plan.set_measured(meas)
    model = (1e-3 * torch.randn((G * G, 2), device=dev, generator=gen)).contiguous()
    res = torch.empty_like(model)
    t_pass = ev_time(lambda: plan.cycle(model, res, S.SDP_DEGRID_CONV), reps)
    prol = torch.empty(G // 2 + 1, dtype=torch.float32, device=dev)
    D.prolate_table(G, prol)
    psf = torch.empty(G * G, dtype=torch.float32, device=dev)
    psf_max = D.psf_generate(plan, prol, psf)
    del model, res
    torch.cuda.empty_cache()
    pcfg = S.PipelineConfig(G, OS, w.cfg.uv_scale, w.cfg.w_scale, w.cfg.cell_size, 200, 200, 0.1, 1.5, 0.0002,
                            psf_max, S.SDP_DEGRID_CONV, S.SDP_COORD_F32, 0, 1)
    pipe = D.pipeline(pcfg, uvw, meas, psf, wk_g, wk_d, keep=(uvw, gk, dk, sup))
    t_cyc = ev_time(pipe.major_cycle, 2)
    out = {"workload": "512 antennas 40 km spiral, 200 time steps, 26163200 vis, G=8192, 64 w-planes hs=4 "
                       "OS=16 (kernels generated on the GPU)",
           "ms_plan_build": t_plan, "ms_fused_pass": t_pass, "vis_per_s_fused_pass": N / (t_pass * 1e-3),
           "ms_major_cycle": t_cyc, "cuda_graph": pipe.graph_active(), "minor_cycles": 200}
    pipe.close()
    plan.close()
    del psf, meas, uvw
    torch.cuda.empty_cache()
    return out


def unet_flops(n: int, h: int, w: int, base: int = 32, backward: bool = False) -> int:
    """Tensor FLOPs (2 per multiply-add) of the U-Net's 3x3 convolutions and
    head for n images of h x w; backward: the data gradients (all but the
    first layer) plus the weight gradients."""
    shapes = []
    for lv in range(4):
        shapes += [(lv, 32 if lv == 0 else base << (lv - 1), base << lv), (lv, base << lv, base << lv)]
    for lv in range(2, -1, -1):
        shapes += [(lv, (base << lv) + (base << (lv + 1)), base << lv), (lv, base << lv, base << lv)]
    fwd = sum(2 * 9 * ci * co * n * (h >> lv) * (w >> lv) for lv, ci, co in shapes) + 2 * base * n * h * w
    if not backward:
        return fwd
    dgrad = sum(2 * 9 * ci * co * n * (h >> lv) * (w >> lv) for lv, ci, co in shapes[1:])
    return dgrad + (fwd - 2 * base * n * h * w) + 4 * base * n * h * w


def fft_block(S, D, dev, G: int = 2048, reps: int = 20):
    """The 2-D FFT of a G x G complex grid (seeded normal values): the FP32
    Stockham transform and the tensor-core transform (BF16 split hi/lo,
    FP32 accumulation), time per transform (CUDA events, median) and error
    against numpy's complex128 FFT."""
    import torch
    rng = np.random.default_rng(11)
    x = rng.standard_normal((G * G, 2)).astype(np.float32)
    xd = torch.from_numpy(x).to(dev)
    out, work = torch.empty_like(xd), torch.empty_like(xd)

    def ev(fn):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return statistics.median(ts)

    ref = np.fft.fft2((x[:, 0] + 1j * x[:, 1]).astype(np.complex128).reshape(G, G)).reshape(-1)
    res = {"grid": G}
    for name, fn in (("fp32", lambda: D.fft2d(G, xd, out, -1)), ("tensor_bf16x3", lambda: D.fft2d_tc(G, xd, out, -1,
                                                                                                      work))):
        t = ev(fn)
        o = out.cpu().numpy().astype(np.float64)
        err = float(np.linalg.norm((o[:, 0] + 1j * o[:, 1]) - ref) / np.linalg.norm(ref))
        res[name] = {"ms": t, "rel_rms_vs_fp64": err}
    return res


def calibration_block(S, D, dev, cpu_baseline: bool, nrx: int = 256, reps: int = 5):
    """One gain-calibration cycle (gains_calibration_run.c: normal equations,
    SVD, SUQ product, gain update) for nrx receivers, one sample per
    baseline (nrx (nrx - 1) / 2 baselines; 512 x 512 normal matrix at 256):
    the device path (CUDA events, median), the actor path with host buffers
    (wall clock), and the reference's compiled actors on the host with
    numpy's SVD in place of LAPACK's (the reference build has no LAPACK here),
    with the error of the device step's gains against that chain."""
    import ctypes as C
    import torch
    rng = np.random.default_rng(5)
    pairs = np.array([(a, b) for a in range(nrx) for b in range(a + 1, nrx)], np.int32)
    nbl, n = pairs.shape[0], 2 * nrx
    g_true = (1.0 + 0.1 * rng.standard_normal(nrx)) * np.exp(1j * 0.3 * rng.standard_normal(nrx))
    pred = rng.standard_normal(nbl) + 1j * rng.standard_normal(nbl)
    meas = pred * g_true[pairs[:, 0]] * np.conj(g_true[pairs[:, 1]])
    c2 = lambda z: np.ascontiguousarray(np.stack([z.real, z.imag], 1).astype(np.float32))  # noqa: E731
    m2, p2, g0 = c2(meas), c2(pred), c2(np.ones(nrx, complex))
    f32 = dict(dtype=torch.float32, device=dev)
    dm, dp, dg = (torch.from_numpy(a).to(dev) for a in (m2, p2, g0))
    dpairs = torch.from_numpy(pairs).to(dev)
    A, Q, Sv, U, VT, suq = (torch.empty(n * n, **f32), torch.empty(n, **f32), torch.empty(n, **f32),
                            torch.empty(n * n, **f32), torch.empty(n * n, **f32), torch.empty(n, **f32))
    gout = torch.empty_like(dg)
    flags = torch.zeros(1, dtype=torch.int32, device=dev)
    ws = torch.empty(D.svd_workspace_bytes(n), dtype=torch.uint8, device=dev)

    def cycle():
        D.gaincal_normal_equations(dpairs, dm, dp, dg, A, Q, flags)
        D.svd(n, A, Sv, U, VT, ws)
        D.gaincal_suq(n, Sv, U, Q, suq)
        D.gaincal_update(n, suq, VT, dg, gout)

    cycle()
    torch.cuda.synchronize()
    sweeps = D.svd_check(ws)
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        cycle()
        b.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    g_dev = gout.cpu().numpy()
    lib = D.lib
    cfg = S.make_config(64, 1.0, 1.0, 8)
    _i, _p = C.c_int, C.c_void_p
    ptr = lambda a: a.ctypes.data_as(_p)  # noqa: E731

    def actor_chain(l, svd_fn=None):
        Ah, Qh = np.zeros((n, n), np.float32), np.zeros(n, np.float32)
        tok = _i(1)
        l.update_gain_calibration_actor(_i(nbl), _i(nrx), _i(nbl), C.byref(tok), ptr(m2), ptr(p2), ptr(g0),
                                        ptr(pairs), C.byref(cfg), ptr(Ah), ptr(Qh))
        if svd_fn is None:
            Sh, Uh, Vh = np.zeros(n, np.float32), np.zeros((n, n), np.float32), np.zeros((n, n), np.float32)
            l.execute_calibration_SVD_actor(_i(n), _i(n), ptr(Ah), ptr(Sh), ptr(Uh), ptr(Vh))
        else:
            Sh, Uh, Vh = svd_fn(Ah)
        sq = np.zeros(n, np.float32)
        l.calculate_SUQ_product_actor(_i(n), _i(n), ptr(Sh), ptr(Uh), ptr(Qh), C.byref(cfg), ptr(sq))
        go = np.zeros((nrx, 2), np.float32)
        l.calculate_delta_update_gains_actor(_i(n), _i(nrx), ptr(sq), ptr(Vh), C.byref(cfg), ptr(g0), ptr(go))
        return go

    def numpy_svd(Ah):
        u, sv, vt = np.linalg.svd(Ah.astype(np.float64).T)
        return (sv.astype(np.float32), np.ascontiguousarray(u.T).astype(np.float32),
                np.ascontiguousarray(vt.T).astype(np.float32))

    actor_chain(lib)
    t0 = time.perf_counter()
    for _ in range(reps):
        actor_chain(lib)
    t_actor = (time.perf_counter() - t0) / reps * 1e3
    res = {"workload": f"{nrx} receivers, {nbl} baselines, {n} x {n} normal matrix",
           "device_ms": float(statistics.median(ts)), "actor_ms": t_actor, "svd_sweeps": sweeps}
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    if cpu_baseline and O.RefLib.available("f32"):
        ref = O.RefLib("f32").lib
        t0 = time.perf_counter()
        g_ref = actor_chain(ref, numpy_svd)
        try:
            from threadpoolctl import threadpool_info
            blas_threads = max([t.get("num_threads", 1) for t in threadpool_info()] or [1])
        except Exception:
            blas_threads = 1
        res["cpu_baseline"] = {"ms": (time.perf_counter() - t0) * 1e3, "kind": "reference", "cores": blas_threads,
                               "sample": "one cycle: the reference's compiled actors (oracle/_ref, one thread) "
                                         "with numpy.linalg.svd (LAPACK, FP64, the BLAS threads) in place of gesvd"}
        z1, z2 = g_dev[:, 0] + 1j * g_dev[:, 1], g_ref[:, 0] + 1j * g_ref[:, 1]
        z1 = z1 * np.exp(-1j * np.angle(np.vdot(z2, z1)))  # the free common phase
        res["gains_rel_err_vs_reference"] = float(np.abs(z1 - z2).max() / np.abs(z2).max())
    return res


def c4_learned_block(S, D, dev, skies: int):
    """Learned CLEAN proposals against plain Hogbom on held-out skies: one
    channel of the 256-antenna spiral layout (3,916,800 visibilities) imaged
    at 1024^2 (17 w-planes hs=4, kernels generated on the GPU); skies of
    10-500 points and 0-20 Gaussians (seed never used in training).  The
    plain pipeline runs 10 major cycles (200 Hogbom minor cycles, DFT
    predict); the learned one runs until it reaches the plain final FP64
    residual RMS x 1.01.  The same comparison on 8 skies at 2048^2 (same
    layout and cell, twice the field; the network is the one trained at
    1024^2).  Also times the network: forward at 1024^2 and one training
    step (16 crops of 256^2)."""
    import torch
    import learned as L

    img = L.Imaging(D, L.spiral_layout(1024))
    params = L.load_weights()
    rows = L.evaluate(img, params, skies, seed=777)
    sp = [r["plain_s"] / r["learned_s"] for r in rows if r["learned_s"]]
    img2 = L.Imaging(D, L.spiral_layout(2048))
    rows2 = L.evaluate(img2, params, max(1, skies // 2), seed=777)
    img2.close()
    sp2 = [r["plain_s"] / r["learned_s"] for r in rows2 if r["learned_s"]]

    def ev(fn, n=7):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(n):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return statistics.median(ts)

    net = S.UNet(D.lib, L.IN_CHANNELS, 1, 1024, 1024, training=False)
    net.set_params(params)
    x = torch.randn((1, L.IN_CHANNELS, 1024, 1024), device=dev)
    out = torch.empty((1, 1024, 1024), device=dev)
    t_fwd = ev(lambda: net.forward(x, out))
    net.check()
    net.set_tensor_path(False)
    t_fwd_legacy = ev(lambda: net.forward(x, out))
    net.close()
    tn = S.UNet(D.lib, L.IN_CHANNELS, 16, 256, 256, training=True)
    tn.set_params(params)
    xb = torch.randn((16, L.IN_CHANNELS, 256, 256), device=dev)
    ob = torch.empty((16, 256, 256), device=dev)
    gb = 1e-6 * torch.randn_like(ob)

    def step():
        tn.forward(xb, ob)
        tn.zero_grads()
        tn.backward(gb)
        tn.adam_step(0.0)

    t_train = ev(step)
    tn.check()
    tn.close()
    f_fwd = unet_flops(1, 1024, 1024)
    f_train = f_fwd + unet_flops(16, 256, 256, backward=True)
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except (OSError, ValueError):
        pass
    bf16 = peaks.get("bf16_tflops") or 1590.0
    img.close()
    med = lambda xs: float(statistics.median(xs)) if xs else None  # noqa: E731
    return {
        "workload": "256 antennas 10 km spiral, 3916800 vis, G=1024, 17 w-planes hs=4; held-out skies of 10-500 "
                    "points + 0-20 Gaussians (FWHM 2-10 px)",
        "skies": len(rows), "plain": "10 major cycles x 200 Hogbom minor cycles (gain 0.1), DFT predict",
        "target": "plain final FP64 residual RMS x 1.01",
        "speedup_median": med(sp), "speedup_geomean": float(np.exp(np.mean(np.log(sp)))) if sp else None,
        "speedup_min": min(sp) if sp else None, "speedup_max": max(sp) if sp else None,
        "reached": sum(1 for r in rows if r["learned_s"]),
        "plain_ms_median": med([r["plain_s"] * 1e3 for r in rows]),
        "learned_ms_median": med([r["learned_s"] * 1e3 for r in rows if r["learned_s"]]),
        "learned_cycles": [r["learned_cycles"] for r in rows], "learned_kinds": [r["learned_kinds"] for r in rows],
        "at_2048": {"skies": len(rows2), "reached": sum(1 for r in rows2 if r["learned_s"]),
                    "speedup_median": med(sp2),
                    "speedup_geomean": float(np.exp(np.mean(np.log(sp2)))) if sp2 else None,
                    "speedup_min": min(sp2) if sp2 else None,
                    "plain_ms_median": med([r["plain_s"] * 1e3 for r in rows2]),
                    "learned_ms_median": med([r["learned_s"] * 1e3 for r in rows2 if r["learned_s"]]),
                    "learned_kinds": [r["learned_kinds"] for r in rows2]},
        "unet_forward_ms_1024": t_fwd, "unet_forward_tflops": f_fwd / (t_fwd * 1e-3) / 1e12,
        "unet_train_step_ms_16x256": t_train, "unet_train_tflops": f_train / (t_train * 1e-3) / 1e12,
        "unet_frac_of_bf16_peak": f_fwd / (t_fwd * 1e-3) / 1e12 / bf16,
        "tensor_path": "tcgen05.mma (TMEM accumulators, TMA loads, warp-specialised)",
        "unet_forward_ms_1024_mma_sync": t_fwd_legacy,
    }


def b200_arm(args):
    import torch
    import torch.distributed as dist
    import sdp_b200 as S

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    lib = S.load()
    D = S.Device(lib)
    A = S.Actors(lib)
    stream = torch.cuda.current_stream()

    w = workload(rank)
    G, OS, NK = w.cfg.grid_size, w.cfg.oversampling, w.cfg.num_kernels
    N = w.num_vis
    taps = (2 * w.half_support) ** 2

    # ---- device-resident inputs -------------------------------------------------------
    uvw_raw = torch.from_numpy(w.uvw).to(dev)
    uvw = torch.empty_like(uvw_raw)
    D.correct_to_finegrid(G, OS, w.cfg.uv_scale, uvw_raw, uvw)
    gk = torch.from_numpy(w.gkernels).to(dev)
    dk = torch.from_numpy(w.dkernels).to(dev)
    sup = torch.from_numpy(w.supports).to(dev)
    wk_g = S.Device.wkernels(gk, sup, w.supports)
    wk_d = S.Device.wkernels(dk, sup, w.supports)
    # measured visibilities: DFT of the 200-point sky on the GPU plus noise
    sky = torch.from_numpy(w.sky.astype(np.float32)).to(dev)
    measured = torch.empty((N, 2), dtype=torch.float32, device=dev)
    D.dft(sky, uvw, measured)
    gen = torch.Generator(device=dev).manual_seed(17 + rank)
    measured += 1e-4 * torch.randn(measured.shape, device=dev, generator=gen)
    # model: 200 CLEAN-like components on the image, to a model grid
    model_img = torch.zeros(G * G, dtype=torch.float32, device=dev)
    pix = torch.randint(G // 4, 3 * G // 4, (200, 2), device=dev, generator=gen)
    model_img[pix[:, 1] * G + pix[:, 0]] = torch.rand(200, device=dev, generator=gen)
    work = torch.empty((G * G, 2), dtype=torch.float32, device=dev)
    model_grid = torch.empty((G * G, 2), dtype=torch.float32, device=dev)
    D.image_to_grid(G, model_img, work, model_grid)
    residual = torch.empty((G * G, 2), dtype=torch.float32, device=dev)
    # plan shape from the autotuner (tile side, visibilities per work item,
    # lanes per visibility), timed on this workload's own fused pass
    t_tune = time.perf_counter()
    shape, tuned_ms, n_shapes = D.autotune(G, OS, w.cfg.uv_scale, w.cfg.w_scale, uvw, wk_g, wk_d, measured,
                                          model_grid, residual, reps=5)
    tune = {"tile": shape.tile, "chunk": shape.chunk, "lanes": shape.lanes or "from support",
            "ms_per_pass": tuned_ms, "shapes_timed": n_shapes, "seconds": time.perf_counter() - t_tune,
            "default": {"tile": 32, "chunk": 1024}}
    plan = D.plan(G, OS, w.cfg.uv_scale, w.cfg.w_scale, uvw, wk_g, wk_d, keep=(uvw, gk, dk, sup), options=shape)
    plan.set_measured(measured)
    plan.check_flags()
    n_items = plan.num_work_items()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2

    def step():
        plan.cycle(model_grid, residual, S.SDP_DEGRID_CONV)

    clocks = ClockSampler(local).__enter__()
    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    plan.check_flags()

    # ---- timed region (device) ---------------------------------------------------------
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.mark(0)
    for i in range(args.steps):
        flush.zero_()
        starts[i].record(stream)
        step()
        ends[i].record(stream)
    torch.cuda.synchronize()
    clocks.mark(1)
    clocks.__exit__(None, None, None)
    if world > 1:
        dist.barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    t_step = sum(step_ms) / len(step_ms)
    t_step = channels.max_over_ranks(t_step, device=dev)
    value = world * N / (t_step * 1e-3)

    # ---- roofline of the dominant kernel (the fused tile kernel) -----------------------
    alg_bytes = algorithmic_bytes(N, G)
    achieved = alg_bytes / (t_step * 1e-3) / 1e9
    peaks = {}
    pf = ROOT / "MEASURED_PEAKS.json"
    if pf.exists():
        peaks = json.loads(pf.read_text())
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    traffic = read_traffic("k_tiles_cycle_conv_c2_2048")
    # the unit that binds this kernel: the shared-memory data pipe, one
    # wavefront per SM per clock (wavefronts per launch from the committed
    # ncu summary; clock: the median SM clock sampled in the timed region)
    wf = read_profile_value("k_tiles_cycle_conv_c2_2048", "shared_wavefronts_per_launch")
    binding = None

    # ---- whole major cycle (device pipeline, CUDA graph): image->grid, fused
    #      vis pass, grid->image, 200 Hogbom minor cycles ---------------------------------
    major = None
    if not args.no_major_cycle:
        ones = torch.zeros((N, 2), dtype=torch.float32, device=dev)
        ones[:, 0] = 1.0
        pgrid = torch.empty((G * G, 2), dtype=torch.float32, device=dev)
        plan.grid(ones, pgrid)
        prol = torch.empty(G // 2 + 1, dtype=torch.float32, device=dev)
        D.prolate_table(G, prol)
        psf = torch.empty(G * G, dtype=torch.float32, device=dev)
        D.grid_to_image(G, pgrid, prol, work, psf)
        psf_max = float(psf.max().item())
        psf /= psf_max
        del ones, pgrid
        pcfg = S.PipelineConfig(G, OS, w.cfg.uv_scale, w.cfg.w_scale, w.cfg.cell_size, 200, 200, 0.1, 1.5, 0.0002,
                                psf_max, S.SDP_DEGRID_CONV, S.SDP_COORD_F32, 0, 1)
        pl = D.pipeline(pcfg, uvw, measured, psf, wk_g, wk_d, keep=(uvw, gk, dk, sup))
        for _ in range(2):
            pl.major_cycle()
        torch.cuda.synchronize()
        n_cyc = max(2, min(5, args.steps))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n_cyc):
            pl.major_cycle()
        e1.record(stream)
        torch.cuda.synchronize()
        t_cyc = e0.elapsed_time(e1) / n_cyc
        major = {"ms_per_major_cycle": t_cyc, "vis_per_s": N / (t_cyc * 1e-3), "minor_cycles": 200,
                 "cuda_graph": pl.graph_active(), "graph_error": pl.graph_error(),
                 "stages": "image->grid FFT, fused degrid/subtract/grid, grid->image FFT + taper, Hogbom x200"}
        pl.close()
        # time to the target residual RMS (plain Hogbom pipeline): from an empty
        # model, cycles until the FP64 residual RMS is within 1 % of the lowest
        # reached in 12 cycles
        pl = D.pipeline(pcfg, uvw, measured, psf, wk_g, wk_d, keep=(uvw, gk, dk, sup))
        ms, rms = [], []
        for _ in range(12):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            pl.major_cycle()
            e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
            rms.append(pl.residual_rms())
        target = 1.01 * min(rms)
        k = next(i for i, r in enumerate(rms) if r <= target)
        major["time_to_rms"] = {"target": "1.01 x the lowest FP64 residual RMS of 12 plain cycles",
                                "cycles": k + 1, "ms": float(sum(ms[:k + 1])),
                                "rms_per_cycle": [float(r) for r in rms],
                                "learned": "c4_learned (the reference's FFT-pipeline prediction does not converge; "
                                           "the learned comparison runs on the DFT-predict major cycle)"}
        pl.close()

    # ---- the batched multi-channel pass (one GPU only) ---------------------------------
    c3 = None
    if world == 1 and not args.no_c3:
        c3 = c3_block(S, D, dev)

    c5 = None
    if world == 1 and not args.no_c5:
        c5 = c5_block(S, D, dev)

    c4 = None
    if world == 1 and not args.no_c4:
        c4 = c4_learned_block(S, D, dev, args.c4_skies)
    fftc = fft_block(S, D, dev) if world == 1 and not args.no_c4 else None
    calib = calibration_block(S, D, dev, not args.no_cpu_baseline) if world == 1 and not args.no_c4 else None

    # ---- e2e through the reference-facing C ABI with pinned host buffers ---------------
    uvw_h = torch.empty((N, 3), dtype=torch.float32).pin_memory()
    uvw_h.copy_(uvw.cpu())
    meas_h = torch.empty((N, 2), dtype=torch.float32).pin_memory()
    meas_h.copy_(measured.cpu())
    mgrid_h = torch.empty((G * G, 2), dtype=torch.float32).pin_memory()
    mgrid_h.copy_(model_grid.cpu())
    pred_h = torch.empty((N, 2), dtype=torch.float32).pin_memory()
    delta_h = torch.empty((N, 2), dtype=torch.float32).pin_memory()
    grid_h = torch.empty((G * G, 2), dtype=torch.float32).pin_memory()
    gk_h, dk_h, sup_h = w.gkernels, w.dkernels, w.supports
    cfg = S.make_config(G, w.cfg.uv_scale, w.cfg.w_scale, OS)
    uvw_n, meas_n, mgrid_n = uvw_h.numpy(), meas_h.numpy(), mgrid_h.numpy()
    pred_n, delta_n, grid_n = pred_h.numpy(), delta_h.numpy(), grid_h.numpy()
    A.set_degrid_mode(S.SDP_DEGRID_CONV)

    def e2e_step():
        A.std_degridding(cfg, G, OS, dk_h, sup_h, mgrid_n, uvw_n, out=pred_n)
        A.subtract_finegrid(meas_n, pred_n, out=delta_n)
        A.std_gridding(cfg, G, OS, gk_h, sup_h, uvw_n, delta_n, out=grid_n)

    e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        e2e_step()
    t_e2e = (time.perf_counter() - t0) / args.e2e_steps
    t_e2e_t = torch.tensor([t_e2e], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t_e2e_t, op=dist.ReduceOp.MAX)
    t_e2e = float(t_e2e_t.item())
    A.set_degrid_mode(S.SDP_DEGRID_NEAREST)
    ksz = gk_h.nbytes + sup_h.nbytes
    h2d = (N * 12 + G * G * 8 + ksz) + (2 * N * 8) + (ksz + N * 12 + N * 8)
    d2h = N * 8 + N * 8 + G * G * 8

    # ---- CPU baseline (rank 0, N = 1) --------------------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = cpu_threads()
        sample = max(threads * 2000, args.cpu_sample)
        t_cpu, kind = cpu_reference_pass(w, uvw_h.numpy(), mgrid_n, sample, threads)
        cpu = {"value": sample / t_cpu, "unit": UNIT, "cores": threads, "kind": kind,
               "sample": f"{sample} visibilities of the workload, {threads} slices on {threads} threads"}

    csum = clocks.summary()
    if wf is not None and csum.get("sm_mhz"):
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        peak_wf = sms * float(csum["sm_mhz"]) * 1e6
        ach_wf = wf / (t_step * 1e-3)
        binding = {"unit": "shared-memory wavefronts/s", "achieved": ach_wf, "peak": peak_wf,
                   "frac": ach_wf / peak_wf, "per_launch": wf,
                   "peak_source": f"{sms} SMs x 1 wavefront/clock x median SM clock in the timed region",
                   "note": "the fused pass is bound by the L1/shared-memory pipe (emulated float atomics, "
                           "bank conflicts), not HBM; see profiles/k_tiles_cycle_conv_c2_2048.txt"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": t_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{w.name}: 256 antennas, 10 km log spiral, 120 time steps, {N} vis per channel, "
                               f"G=2048, 17 w-planes hs=4 OS=16, one channel per GPU",
                   "degrid": "convolutional (normalised, degridgrid.c:147-191)",
                   "l2": "flushed between timed steps (256 MB write)", "work_items": n_items,
                   "plan_shape": tune},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                     "kernel": "k_tiles<STD, OP_CYCLE_CONV>",
                     "algorithmic_bytes_per_launch": alg_bytes,
                     "fp32_flops_per_launch": algorithmic_flops(N, taps)},
        "roofline_binding": binding,
        "e2e": {"value": world * N / t_e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "path": "std_degridding + subtract_from_measurements_finegrid + std_gridding (host buffers)"},
        "gpu_launches": args.steps,
        "clocks": csum,
    }
    if major is not None:
        line["major_cycle"] = major
    if c3 is not None:
        line["c3_batched"] = c3
    if c5 is not None:
        line["c5_channel_8192"] = c5
    if c4 is not None:
        line["c4_learned"] = c4
    if fftc is not None:
        line["fft_2048"] = fftc
    if calib is not None:
        line["gain_calibration"] = calib
    if cpu is not None:
        line["cpu_baseline"] = cpu
    plan.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    return b200_arm(args)


if __name__ == "__main__":
    sys.exit(main())
