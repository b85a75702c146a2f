"""Benchmark: visibilities gridded + degridded per second on B200.

One step = one major-cycle visibility pass over every visibility of the
largest configuration (the 8192^2 workload): 512 antennas on a seeded 40 km
log spiral, 16 channels over 100-200 MHz x 200 time steps, 16 x 26,163,200 =
418,611,200 visibilities, one 8192^2 grid per channel, 64 w-planes of half
support 4 (kernels generated on the GPU), oversampling 16.  Per visibility:
W-projection degridding of the model grid (convolutional,
degridgrid.c:147-191), subtraction from the measured value
(gains_apply_run.c:273-297) and gridding of the residual
(degridgrid.c:69-125); all channels in one persistent batched launch
(sdp_visbatch).  Measured visibilities: the exact DFT of a seeded sky of
1000 points and 50 Gaussians plus noise (no public dataset is used).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

value: device-resident throughput (inputs in HBM, several GB, larger than
L2; L2 also flushed between timed steps; CUDA events; max over ranks).
Under torchrun the 16 channels are dealt to the ranks by visibility count
(strong scaling: the total work is fixed); N > 1 adds the continuum exchange
step (each rank sums its channels' residual grids, then one NCCL
all-reduce).  e2e: the same pass through the reference-facing C ABI
(std_degridding, subtract_from_measurements_finegrid, std_gridding per
channel) with pinned host buffers and the host<->device copies inside the
timed region.  --impl reference times the reference's own actor code
compiled from its sources (oracle/_ref) on the host cores, on the same
workload, over a stated per-channel sample.  Other blocks of the line: the
single 2048^2 channel (3.9 M visibilities), the graph-captured major cycle
with Hogbom, the 64-channel batch, learned proposals, the FFTs and gain
calibration.
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
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-major-cycle", action="store_true")
    ap.add_argument("--no-c2", action="store_true", help="skip the single 2048^2 channel block")
    ap.add_argument("--no-c3", action="store_true", help="skip the batched 64-channel pass")
    ap.add_argument("--no-c4", action="store_true", help="skip the learned-proposal comparison")
    ap.add_argument("--no-extras", action="store_true", help="headline only (no FFT / calibration blocks)")
    ap.add_argument("--c4-skies", type=int, default=100, help="held-out skies of the learned-proposal comparison")
    ap.add_argument("--c5-skies", type=int, default=2, help="held-out skies of the 8192^2 learned comparison")
    ap.add_argument("--c2-only", action="store_true", help="only the single 2048^2 channel block (profiling)")
    ap.add_argument("--c2-shape", default="", help="tile,chunk,lanes,warps for the 2048^2 block (no autotune)")
    ap.add_argument("--channels", type=int, default=C5_CHANNELS,
                    help="headline on the first K of the 16 channels (profiling captures of a few GB)")
    ap.add_argument("--cpu-sample", type=int, default=1_000_000,
                    help="visibilities per channel per step of the reference arm / CPU baseline")
    return ap.parse_args()


# The 8192^2 workload: 512 antennas, 40 km log spiral, 200 time steps per
# channel, 16 channels evenly spaced over 100-200 MHz.
C5_CHANNELS = 16
C5_F_LO, C5_F_HI = 100e6, 200e6
C5_GRID, C5_PLANES, C5_HS, C5_OS = 8192, 64, 4, 16


def c5_frequencies():
    return [C5_F_LO + (C5_F_HI - C5_F_LO) * c / (C5_CHANNELS - 1) for c in range(C5_CHANNELS)]


def c5_base():
    """uvw of the top channel (200 MHz; the others are scaled copies, uvw in
    wavelengths is proportional to frequency), the imaging geometry (cell
    chosen so the longest baseline at 200 MHz reaches 0.9 of the half grid)
    and the host kernel tables the reference arm uses."""
    return synth.make_workload("c5_8192", 512, 20000.0, "spiral", 200, C5_GRID, 1, 1e-3, 1.0, 1e-4, C5_PLANES,
                               C5_HS, C5_OS, freq_hz=C5_F_HI, seed=5, compute_vis=False)


def c5_sky(cell: float, G: int, seed: int = 55):
    """1000 points (log-uniform 1e-3-1 Jy) and 50 circular Gaussians (FWHM
    2-10 pixels, log-uniform 1e-2-1 Jy) in the central half of the field, as
    (l, m, flux, sigma) rows for sdp_dft_gauss."""
    rng = np.random.default_rng(seed)
    fov = cell * G
    half = 0.25 * fov
    pts = np.zeros((1000, 4))
    pts[:, :2] = rng.uniform(-half, half, (1000, 2))
    pts[:, 2] = np.exp(rng.uniform(math.log(1e-3), 0.0, 1000))
    gau = np.zeros((50, 4))
    gau[:, :2] = rng.uniform(-half, half, (50, 2))
    gau[:, 2] = np.exp(rng.uniform(math.log(1e-2), 0.0, 50))
    gau[:, 3] = np.exp(rng.uniform(math.log(2.0), math.log(10.0), 50)) * cell / (2.0 * math.sqrt(2.0 * math.log(2.0)))
    return np.concatenate([pts, gau]).astype(np.float32)


def snap_uvw_host(uvw: np.ndarray, G: int, OS: int, us: float) -> np.ndarray:
    """Fine-grid snap of the uvw (degridgrid.c:24-25, 52-54) in numpy with the
    reference's rounding (the reference arm's inputs)."""
    u = uvw.astype(np.float64)
    fx = np.trunc((u[:, 0] * us + G // 2) * OS + 0.5)
    fy = np.trunc((u[:, 1] * us + G // 2) * OS + 0.5)
    out = np.empty_like(uvw)
    out[:, 0] = ((fx / OS - G // 2) / us).astype(np.float32)
    out[:, 1] = ((fy / OS - G // 2) / us).astype(np.float32)
    out[:, 2] = uvw[:, 2]
    return out


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
def cpu_threads() -> int:
    """Host threads for the reference arm: every core, up to 64."""
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    return max(1, min(64, n))


class ReferencePass:
    """The reference's own actors (compiled from its sources, oracle/_ref;
    the oracle restatement when that build is absent) on the host cores over
    a per-channel sample of the 8192^2 workload: per channel one
    std_degridding (as shipped: the kernel sum is computed and then replaced
    by the nearest cell, degridgrid.c:193-200), subtract_from_measurements
    and std_gridding into the channel's own grid (cleared by the reference,
    degridgrid.c:73) -- the calls one channel's PREESM firing makes.  The
    channels run on parallel host threads (up to one per channel); the model
    grid is padded once outside the timed region."""

    def __init__(self, base, sample_per_channel: int, threads: int, seed: int = 77):
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O
        self.O = O
        G, OS, us, ws = base.cfg.grid_size, base.cfg.oversampling, base.cfg.uv_scale, base.cfg.w_scale
        self.G, self.OS = G, OS
        self.cfg = O.make_config(G, us, ws, OS)
        if O.RefLib.available("f32", "fast"):
            self.lib, self.kind = O.RefLib("f32", "fast"), "reference"
        elif O.RefLib.available("f32"):
            self.lib, self.kind = O.RefLib("f32"), "reference"
        else:
            self.lib, self.kind = None, "port"
            self.o = O.Oracle("f32")
        self.base = base
        self.threads = max(1, min(threads, C5_CHANNELS))
        rng = np.random.default_rng(seed)
        self.sample = min(sample_per_channel, base.num_vis)
        model = (rng.standard_normal((G * G, 2)) * 1e-3).astype(np.float32)
        self.model = self.lib.padded_grid(G, model) if self.lib else model
        self.uvw, self.vis = [], []
        for c, f in enumerate(c5_frequencies()):
            idx = np.sort(rng.choice(base.num_vis, self.sample, replace=False))
            u = base.uvw[idx] * np.float32(f / C5_F_HI)
            self.uvw.append(snap_uvw_host(u, G, OS, us))
            self.vis.append((0.1 * rng.standard_normal((self.sample, 2))).astype(np.float32))
        self.grids = [np.empty((G * G, 2), np.float32) for _ in range(self.threads)]

    def _channel(self, c: int, t: int, n: int):
        b, G, OS = self.base, self.G, self.OS
        u = self.uvw[c][:n]
        v = self.vis[c][:n]
        if self.lib is not None:
            p = self.lib.std_degridding(self.cfg, G, OS, b.dkernels, b.supports, self.model, u, padded=True)
            d = self.lib.subtract_finegrid(v, p)
            self.lib.std_gridding(self.cfg, G, OS, b.gkernels, b.supports, u, d, out=self.grids[t])
        else:
            o = self.o
            p = o.std_degridding(G, OS, b.dkernels, b.supports, self.model, u, b.cfg.uv_scale, b.cfg.w_scale, False)
            d = o.subtract_vis(v, p)
            self.grids[t][:] = o.std_gridding(G, OS, b.gkernels, b.supports, u, d, b.cfg.uv_scale, b.cfg.w_scale)

    def run(self, n: int | None = None) -> float:
        """One step over all 16 channels (n visibilities each); seconds."""
        n = self.sample if n is None else min(n, self.sample)

        def worker(t):
            for c in range(t, C5_CHANNELS, self.threads):
                self._channel(c, t, n)

        # silence the reference's progress printf
        devnull = os.open(os.devnull, os.O_WRONLY)
        saved = os.dup(1)
        sys.stdout.flush()
        os.dup2(devnull, 1)
        try:
            t0 = time.perf_counter()
            with ThreadPoolExecutor(max_workers=self.threads) as ex:
                list(ex.map(worker, range(self.threads)))
            t1 = time.perf_counter()
        finally:
            sys.stdout.flush()
            os.dup2(saved, 1)
            os.close(saved)
            os.close(devnull)
        return t1 - t0

    def describe(self) -> str:
        return (f"{self.sample} visibilities of each of the 16 channels per step ({C5_CHANNELS * self.sample} in "
                f"all, a {self.sample / self.base.num_vis:.3f} sample), one std_degridding + subtract + std_gridding "
                f"call per channel, {self.threads} host threads")


def c5_config_name(n_vis_total: int) -> str:
    return (f"c5_8192: 512 antennas, 40 km log spiral, 16 channels 100-200 MHz x 200 time steps, "
            f"{n_vis_total} vis, G=8192 per channel, 64 w-planes hs=4 OS=16")


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    base = c5_base()
    threads = cpu_threads()
    ref = ReferencePass(base, args.cpu_sample, threads)
    for _ in range(max(0, args.warmup)):
        ref.run(20_000)
    times = [ref.run() for _ in range(args.steps)]
    t = statistics.mean(times)
    nvis = C5_CHANNELS * ref.sample
    value = nvis / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": c5_config_name(C5_CHANNELS * base.num_vis),
                   "degrid": "the reference's std_degridding as shipped: kernel sum computed, then replaced by "
                             "the nearest cell (degridgrid.c:193-200)",
                   "sample": ref.describe()},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": ref.threads, "kind": ref.kind,
                         "sample": ref.describe()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


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


class C5Device:
    """The 8192^2 workload's channels owned by this rank on the device: the
    W-projection kernels generated on the GPU, per channel the scaled and
    snapped uvw, measured visibilities (exact DFT of the sky + 0.1 mJy noise)
    and a visibility plan of the autotuned shape (tuned on the top channel,
    the widest uv coverage), all channels in one sdp_visbatch; one shared
    model grid (the model image is channel independent; its grid is too) and
    one residual grid per channel."""

    def __init__(self, S, D, dev, base, owned, tune: bool = True, keep_host: bool = True, shape=None):
        import torch
        self.S, self.D, self.dev = S, D, dev
        G, OS = base.cfg.grid_size, base.cfg.oversampling
        us, ws, cell = base.cfg.uv_scale, base.cfg.w_scale, base.cfg.cell_size
        self.G, self.OS, self.owned, self.cell = G, OS, list(owned), cell
        fov = cell * G
        self.gk, self.dk, self.sup = D.wkernels_generate([C5_HS] * C5_PLANES, OS, base.cfg.max_w, fov)
        self.sup_h = self.sup.cpu().numpy()
        self.wk_g = S.Device.wkernels(self.gk, self.sup, self.sup_h)
        self.wk_d = S.Device.wkernels(self.dk, self.sup, self.sup_h)
        sky = torch.from_numpy(c5_sky(cell, G)).to(dev)
        gen = torch.Generator(device=dev).manual_seed(23)
        # model grid: half the flux of the 1000 points on their pixels, to a grid
        img = torch.zeros(G * G, dtype=torch.float32, device=dev)
        px = torch.round(sky[:1000, :2] / cell).long() + G // 2
        img.index_put_((px[:, 1] * G + px[:, 0],), 0.5 * sky[:1000, 2], accumulate=True)
        work = torch.empty((G * G, 2), dtype=torch.float32, device=dev)
        self.model = torch.empty((G * G, 2), dtype=torch.float32, device=dev)
        D.image_to_grid(G, img, work, self.model)
        del img, work
        uvw_top = torch.from_numpy(base.uvw).to(dev)
        freqs = c5_frequencies()
        self.resid = torch.empty((max(1, len(owned)), G * G, 2), dtype=torch.float32, device=dev)
        self.shape = shape
        self.tune = None
        self.plans, self.counts, self.host = [], [], []
        order = sorted(owned, key=lambda c: -freqs[c])  # the top channel first (autotuned on)
        built = {}
        for c in order:
            uvw_raw = (uvw_top * (freqs[c] / C5_F_HI)).contiguous()
            uvw = torch.empty_like(uvw_raw)
            D.correct_to_finegrid(G, OS, us, uvw_raw, uvw)
            meas = torch.empty((uvw.shape[0], 2), dtype=torch.float32, device=dev)
            D.dft_gauss(sky, uvw_raw, meas)
            meas += 1e-4 * torch.randn(meas.shape, device=dev, generator=gen)
            del uvw_raw
            if tune and self.shape is None:
                t0 = time.perf_counter()
                shape, ms, n = D.autotune(G, OS, us, ws, uvw, self.wk_g, self.wk_d, meas, self.model, self.resid[0],
                                          reps=3)
                self.shape = shape
                self.tune = {"tile": shape.tile, "chunk": shape.chunk, "lanes": shape.lanes, "warps": shape.warps,
                             "ms_per_pass_one_channel": ms, "shapes_timed": n, "seconds": time.perf_counter() - t0,
                             "tuned_on": f"channel {c} ({freqs[c] / 1e6:.1f} MHz)"}
            pl = D.plan(G, OS, us, ws, uvw, self.wk_g, self.wk_d, keep=(self.gk, self.dk, self.sup),
                        options=self.shape)
            pl.set_measured(meas)
            host = (uvw.cpu().numpy(), meas.cpu().numpy()) if keep_host else None
            built[c] = (pl, int(uvw.shape[0]), host)
            del uvw, meas
        del uvw_top
        for c in self.owned:
            pl, n, host = built[c]
            self.plans.append(pl)
            self.counts.append(n)
            self.host.append(host)
        torch.cuda.synchronize()
        for pl in self.plans:
            pl.check_flags()
        self.batch = D.batch(self.plans) if self.plans else None
        if self.batch is not None:
            self.batch.set_grids([self.model] * len(self.plans), [self.resid[k] for k in range(len(self.plans))])
        self.num_vis = sum(self.counts)

    def cycle(self):
        if self.batch is not None:
            self.batch.cycle(self.S.SDP_DEGRID_CONV)

    def close(self):
        if self.batch is not None:
            self.batch.close()
        for pl in self.plans:
            pl.close()
        self.plans = []


def c5_major_cycle_block(S, D, dev, c5: "C5Device", reps: int = 2):
    """One channel of the 8192^2 workload through the whole device major
    cycle (image -> grid FFT, fused pass, grid -> image FFT + taper, 200
    Hogbom minor cycles; CUDA graph): time per cycle."""
    import torch
    k = len(c5.owned) - 1
    pl = c5.plans[k]
    G, OS = c5.G, c5.OS
    uvw_h, meas_h = c5.host[k]
    uvw = torch.from_numpy(uvw_h).to(dev)
    meas = torch.from_numpy(meas_h).to(dev)
    prol = torch.empty(G // 2 + 1, dtype=torch.float32, device=dev)
    D.prolate_table(G, prol)
    psf = torch.empty(G * G, dtype=torch.float32, device=dev)
    psf_max = D.psf_generate(pl, prol, psf)
    geom = pl.geom
    pcfg = S.PipelineConfig(G, OS, geom.uv_scale, geom.w_scale, c5.cell, 200, 200, 0.1, 1.5, 0.0002, psf_max,
                            S.SDP_DEGRID_CONV, S.SDP_COORD_F32, 0, 1)
    pipe = D.pipeline(pcfg, uvw, meas, psf, c5.wk_g, c5.wk_d, keep=(uvw, c5.gk, c5.dk, c5.sup))
    pipe.major_cycle()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        pipe.major_cycle()
        b.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    out = {"channel": c5.owned[k], "vis": int(uvw.shape[0]), "ms_major_cycle": float(statistics.median(ts)),
           "cuda_graph": pipe.graph_active(), "minor_cycles": 200,
           "stages": "image->grid FFT, fused degrid/subtract/grid, grid->image FFT + taper, Hogbom x200"}
    pipe.close()
    del psf, uvw, meas
    torch.cuda.empty_cache()
    return out


def c5_learned_block(S, D, dev, base, shape, skies: int = 2):
    """Learned proposals against plain Hogbom on the 8192^2 workload: all 16
    channels imaged into one continuum image (learned.ContinuumImaging), sky
    of 1000 points + 50 Gaussians (FWHM 2-10 px) per held-out seed, DFT
    predict, 200 Hogbom minor cycles per plain major cycle (10 cycles); the
    learned pipeline (the network trained at 1024^2 on the 10 km array,
    proposals verified by an exact predict/grid cycle, Hogbom fallback) runs
    until the plain final FP64 residual RMS x 1.01."""
    import torch
    import learned as L
    G, cell = base.cfg.grid_size, base.cfg.cell_size
    chans = [np.ascontiguousarray(base.uvw * np.float32(f / C5_F_HI)) for f in c5_frequencies()]
    opts = S.PlanOptions(shape["tile"], shape["chunk"], shape["lanes"], shape["warps"]) if shape else None
    t0 = time.perf_counter()
    img = L.ContinuumImaging(D, chans, G, cell, base.cfg.max_w, num_planes=C5_PLANES, half_support=C5_HS,
                             oversampling=C5_OS, options=opts)
    setup_s = time.perf_counter() - t0
    del chans
    sampler = L.SkySampler(G, cell, seed=991, points=(1000, 1000), gaussians=(50, 50))
    c5w = L.WEIGHTS_C5.exists()
    rows = L.evaluate(img, L.load_weights(L.WEIGHTS_C5 if c5w else L.WEIGHTS), skies, seed=991, sampler=sampler,
                      max_components=512)
    img.close()
    torch.cuda.empty_cache()
    sp = [r["plain_s"] / r["learned_s"] for r in rows if r["learned_s"]]
    return {"workload": "16 channels 100-200 MHz continuum, 418611200 vis, G=8192, 64 w-planes hs=4; held-out skies "
                        "of 1000 points + 50 Gaussians (FWHM 2-10 px)",
            "skies": len(rows), "reached": len(sp), "setup_s": setup_s,
            "network": ("weights/unet_c5.npz: trained on the 40 km array's 16-channel continuum (2048^2 images with "
                        "this cell, every 8th time step)") if c5w else "weights/unet_c4.npz (10 km array, 1024^2)",
            "plain": "10 major cycles x 200 Hogbom minor cycles (gain 0.1), DFT predict over all channels",
            "target": "plain final FP64 residual RMS x 1.01",
            "speedup": sp, "speedup_median": float(statistics.median(sp)) if sp else None,
            "rows": [{k: r[k] for k in ("plain_s", "learned_s", "learned_cycles", "learned_kinds", "rms0",
                                        "plain_final", "learned_final", "plain_rms", "learned_rms")}
                     for r in rows]}


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
        "slower_than_plain": sum(1 for x in sp if x < 1.0),
        "speedup_per_sky": [round(r["plain_s"] / r["learned_s"], 3) if r["learned_s"] else None for r in rows],
        "plain_ms_median": med([r["plain_s"] * 1e3 for r in rows]),
        "learned_ms_median": med([r["learned_s"] * 1e3 for r in rows if r["learned_s"]]),
        "learned_cycles": [r["learned_cycles"] for r in rows], "learned_kinds": [r["learned_kinds"] for r in rows],
        "learned_rms_ratio": [[round(b / a, 3) for a, b in zip([r["rms0"]] + r["learned_rms"][:-1], r["learned_rms"])]
                              for r in rows],
        "plain_rms_ratio": [[round(b / a, 3) for a, b in zip([r["rms0"]] + r["plain_rms"][:-1], r["plain_rms"])]
                            for r in rows[:8]],
        "at_2048": {"skies": len(rows2), "reached": sum(1 for r in rows2 if r["learned_s"]),
                    "speedup_median": med(sp2),
                    "speedup_geomean": float(np.exp(np.mean(np.log(sp2)))) if sp2 else None,
                    "speedup_min": min(sp2) if sp2 else None,
                    "slower_than_plain": sum(1 for x in sp2 if x < 1.0),
                    "plain_ms_median": med([r["plain_s"] * 1e3 for r in rows2]),
                    "learned_ms_median": med([r["learned_s"] * 1e3 for r in rows2 if r["learned_s"]]),
                    "learned_kinds": [r["learned_kinds"] for r in rows2]},
        "unet_forward_ms_1024": t_fwd, "unet_forward_tflops": f_fwd / (t_fwd * 1e-3) / 1e12,
        "unet_train_step_ms_16x256": t_train, "unet_train_tflops": f_train / (t_train * 1e-3) / 1e12,
        "unet_frac_of_bf16_peak": f_fwd / (t_fwd * 1e-3) / 1e12 / bf16,
        "tensor_path": "tcgen05.mma (TMEM accumulators, TMA loads, warp-specialised)",
        "unet_forward_ms_1024_mma_sync": t_fwd_legacy,
    }


def peaks_block(D, dev) -> dict:
    """On-chip ceilings measured on this GPU (sdp_peak_measure): L2 reads of a
    32 MB buffer, conflict-free shared-memory reads, scalar and packed FP32
    FMA, and the rate of the Hogbom residual update in the reference's types."""
    import torch
    scratch = torch.zeros(32 << 20, dtype=torch.uint8, device=dev)
    r = {k: D.peak(k, scratch, reps=10) for k in D.PEAK_KINDS}
    del scratch
    return {"l2_read_gbs": r["l2_read"] / 1e9, "smem_read_gbs": r["smem_read"] / 1e9,
            "fp32_fma_tflops": r["fp32_fma"] / 1e12, "fp32x2_fma_tflops": r["fp32x2_fma"] / 1e12,
            "hogbom_update_gpix_s": r["hogbom_update"] / 1e9,
            "method": "csrc/peaks.cu: one kernel per ceiling, 4 x 512 threads per SM, 10 launches after one "
                      "warm-up, CUDA events"}


def hogbom_block(S, D, dev, G, dirty, psf, psf_max, cell, peaks, reps=5):
    """Hogbom alone (sdp_hogbom, 200 minor cycles, gain 0.1) on a dirty image:
    time per minor cycle, and the PSF pass against the measured L2 read and
    residual-update ceilings.  The pass reads, per minor cycle, the PSF window
    the component's position selects (deconvolution_run.c:264-272): 4 bytes of
    PSF and one update per pixel of the window."""
    import torch
    prm = S.CleanParams(G, 200, 200, 0.1, 1.5, 0.0002, psf_max, cell)
    ws = torch.empty(max(1, D.hogbom_workspace_bytes(G)), dtype=torch.uint8, device=dev)
    res = torch.empty_like(dirty)
    model = torch.zeros_like(dirty)
    src = torch.zeros((200, 3), dtype=torch.float32, device=dev)
    cnt = torch.zeros(1, dtype=torch.int32, device=dev)
    ts = []
    for i in range(reps + 2):
        res.copy_(dirty)
        model.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        D.hogbom(prm, res, psf, model, src, cnt, ws)
        b.record()
        torch.cuda.synchronize()
        if i >= 2:
            ts.append(a.elapsed_time(b))
    n = int(cnt.item())
    t = float(statistics.median(ts))
    h = G // 2
    pix = 0
    for x, y, _ in src[:n].cpu().numpy().astype(np.float64):
        mx, my = int(round(x / cell)) + h, int(round(y / cell)) + h
        pix += (min(mx, h) + min(G - mx, h)) * (min(my, h) + min(G - my, h))
    out = {"grid": G, "minor_cycles": n, "ms": t, "us_per_minor_cycle": t * 1e3 / max(n, 1),
           "window_pixels_per_minor_cycle": pix / max(n, 1),
           "psf_l2_gbs": 4.0 * pix / (t * 1e-3) / 1e9,
           "updates_gpix_s": pix / (t * 1e-3) / 1e9}
    if peaks:
        out["psf_l2_frac_of_measured"] = out["psf_l2_gbs"] / peaks["l2_read_gbs"]
        out["update_frac_of_measured"] = out["updates_gpix_s"] / peaks["hogbom_update_gpix_s"]
    return out


def c2_block(S, D, dev, args, clocks_mhz=None):
    """The single 2048^2 channel (256 antennas, 10 km log spiral, 120 time
    steps: 3,916,800 visibilities; 17 w-planes hs=4, OS 16): the fused pass
    with the autotuned plan shape (CUDA events, L2 flushed between passes),
    its roofline figures, the graph-captured major cycle with 200 Hogbom
    minor cycles, and the time to the plain pipeline's lowest residual RMS."""
    import torch
    stream = torch.cuda.current_stream()
    w = synth.make_workload("c2_2048", 256, 5000.0, "spiral", 120, 2048, 200, 1e-3, 1.0, 1e-4, 17, 4,
                            freq_hz=140e6, seed=2, compute_vis=False)
    G, OS, N = w.cfg.grid_size, w.cfg.oversampling, w.num_vis
    uvw_raw = torch.from_numpy(w.uvw).to(dev)
    uvw = torch.empty_like(uvw_raw)
    D.correct_to_finegrid(G, OS, w.cfg.uv_scale, uvw_raw, uvw)
    gk = torch.from_numpy(w.gkernels).to(dev)
    dk = torch.from_numpy(w.dkernels).to(dev)
    sup = torch.from_numpy(w.supports).to(dev)
    wk_g = S.Device.wkernels(gk, sup, w.supports)
    wk_d = S.Device.wkernels(dk, sup, w.supports)
    sky = torch.from_numpy(w.sky.astype(np.float32)).to(dev)
    measured = torch.empty((N, 2), dtype=torch.float32, device=dev)
    D.dft(sky, uvw, measured)
    gen = torch.Generator(device=dev).manual_seed(17)
    measured += 1e-4 * torch.randn(measured.shape, device=dev, generator=gen)
    model_img = torch.zeros(G * G, dtype=torch.float32, device=dev)
    pix = torch.randint(G // 4, 3 * G // 4, (200, 2), device=dev, generator=gen)
    model_img[pix[:, 1] * G + pix[:, 0]] = torch.rand(200, device=dev, generator=gen)
    work = torch.empty((G * G, 2), dtype=torch.float32, device=dev)
    model_grid = torch.empty((G * G, 2), dtype=torch.float32, device=dev)
    D.image_to_grid(G, model_img, work, model_grid)
    residual = torch.empty((G * G, 2), dtype=torch.float32, device=dev)
    t_tune = time.perf_counter()
    if args.c2_shape:
        shape, tuned_ms, n_shapes = S.PlanOptions(*[int(x) for x in args.c2_shape.split(",")]), None, 0
    else:
        shape, tuned_ms, n_shapes = D.autotune(G, OS, w.cfg.uv_scale, w.cfg.w_scale, uvw, wk_g, wk_d, measured,
                                              model_grid, residual, reps=5)
    tune = {"tile": shape.tile, "chunk": shape.chunk, "lanes": shape.lanes, "warps": shape.warps,
            "ms_per_pass": tuned_ms, "shapes_timed": n_shapes, "seconds": time.perf_counter() - t_tune}
    plan = D.plan(G, OS, w.cfg.uv_scale, w.cfg.w_scale, uvw, wk_g, wk_d, keep=(uvw, gk, dk, sup), options=shape)
    plan.set_measured(measured)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    for _ in range(3):
        plan.cycle(model_grid, residual, S.SDP_DEGRID_CONV)
    torch.cuda.synchronize()
    plan.check_flags()
    ts = []
    for _ in range(max(5, args.steps)):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        plan.cycle(model_grid, residual, S.SDP_DEGRID_CONV)
        b.record(stream)
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    t = statistics.mean(ts)
    taps = (2 * w.half_support) ** 2
    out = {"workload": f"{w.name}: 256 antennas, 10 km log spiral, 120 time steps, {N} vis, G=2048, "
                       f"17 w-planes hs=4 OS=16", "ms_fused_pass": t, "vis_per_s": N / (t * 1e-3),
           "plan_shape": tune, "algorithmic_bytes": algorithmic_bytes(N, G),
           "achieved_gbs": algorithmic_bytes(N, G) / (t * 1e-3) / 1e9,
           "fp32_tflops": algorithmic_flops(N, taps) / (t * 1e-3) / 1e12,
           "traffic": read_traffic("k_vis_fast_cycle_c2_2048")}
    del flush
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
        # Hogbom alone on the dirty image
        dgrid = torch.zeros((G * G, 2), dtype=torch.float32, device=dev)
        plan.grid(measured, dgrid)
        dirty = torch.empty(G * G, dtype=torch.float32, device=dev)
        D.grid_to_image(G, dgrid, prol, work, dirty)
        dirty /= psf_max
        del dgrid
        peaks = getattr(args, "peaks", None)
        out["hogbom"] = hogbom_block(S, D, dev, G, dirty, psf, psf_max, w.cfg.cell_size, peaks)
        del dirty
        if peaks:
            out["fp32_frac_of_measured_fp32x2"] = out["fp32_tflops"] / peaks["fp32x2_fma_tflops"]
        pcfg = S.PipelineConfig(G, OS, w.cfg.uv_scale, w.cfg.w_scale, w.cfg.cell_size, 200, 200, 0.1, 1.5, 0.0002,
                                psf_max, S.SDP_DEGRID_CONV, S.SDP_COORD_F32, 0, 1)
        pl = D.pipeline(pcfg, uvw, measured, psf, wk_g, wk_d, keep=(uvw, gk, dk, sup))
        for _ in range(2):
            pl.major_cycle()
        torch.cuda.synchronize()
        n_cyc = 5
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
                                "rms_per_cycle": [float(r) for r in rms]}
        pl.close()
        out["major_cycle"] = major
    plan.close()
    del work, residual, model_grid, measured, uvw
    torch.cuda.empty_cache()
    return out


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
    args.peaks = peaks_block(D, dev) if world == 1 else None
    if args.c2_only:
        print(json.dumps({"c2_2048": c2_block(S, D, dev, args), "peaks_measured": args.peaks}), flush=True)
        return 0

    # ---- the 8192^2 workload: this rank's channels on the device ---------------------
    base = c5_base()
    G, OS = base.cfg.grid_size, base.cfg.oversampling
    nch = max(1, min(C5_CHANNELS, args.channels))
    counts_all = [base.num_vis] * nch
    owned = channels.assign_channels(counts_all, world)[rank]
    total_vis = int(sum(counts_all))
    t0 = time.perf_counter()
    c5 = C5Device(S, D, dev, base, owned, tune=True, keep_host=True)
    setup_s = time.perf_counter() - t0
    n_items = c5.batch.num_work_items() if c5.batch is not None else 0
    tune = c5.tune
    cont = torch.empty((G * G, 2), dtype=torch.float32, device=dev) if world > 1 else None

    def step():
        c5.cycle()
        if world > 1:  # the continuum exchange: this rank's channel sum, all-reduced
            if c5.plans:
                D.merge_grids(G, len(c5.plans), c5.resid, cont)
            else:
                cont.zero_()
            channels.continuum_sum_(cont)

    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2
    clocks = ClockSampler(local).__enter__()
    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    for pl in c5.plans:
        pl.check_flags()

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
    if world > 1:
        dist.barrier()
    step_ms = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    t_rank = sum(step_ms) / len(step_ms)
    t_step = channels.max_over_ranks(t_rank, device=dev)
    value = total_vis / (t_step * 1e-3)

    # ---- roofline of the dominant kernel: the batched fused pass of this rank --------
    taps = (2 * C5_HS) ** 2
    alg_bytes = sum(algorithmic_bytes(n, G) for n in c5.counts)
    alg_flops = sum(algorithmic_flops(n, taps) for n in c5.counts)
    t_pass = t_rank  # N = 1: the step is the pass (residual-grid clears + one k_vis_fast_batch launch)
    if world > 1:
        ts = []
        for _ in range(3):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            c5.cycle()
            b.record(stream)
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        t_pass = statistics.mean(ts)
    achieved = alg_bytes / (t_pass * 1e-3) / 1e9
    peaks = {}
    pf = ROOT / "MEASURED_PEAKS.json"
    if pf.exists():
        peaks = json.loads(pf.read_text())
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    traffic = read_traffic("k_vis_fast_batch_c5_8192")
    csum = clocks.summary()
    clocks.__exit__(None, None, None)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    sm_mhz = float(csum["sm_mhz"]) if csum.get("sm_mhz") else 1965.0
    pk = getattr(args, "peaks", None)
    if pk:
        fp32_peak = pk["fp32x2_fma_tflops"]
        fp32_src = "measured: packed FP32 FMA (csrc/peaks.cu)"
        peak_wf = pk["smem_read_gbs"] * 1e9 / 128.0
        wf_src = "measured: conflict-free 16-byte shared loads (csrc/peaks.cu), 128 B per wavefront"
    else:
        fp32_peak = sms * 128 * 2 * sm_mhz * 1e6 / 1e12
        fp32_src = f"{sms} SMs x 128 FP32 lanes x 2 x the median SM clock in the timed region"
        peak_wf = sms * sm_mhz * 1e6
        wf_src = f"{sms} SMs x 1 wavefront per clock x the median SM clock"
    binding = {"fp32": {"achieved_tflops": alg_flops / (t_pass * 1e-3) / 1e12, "peak_tflops": fp32_peak,
                        "frac": alg_flops / (t_pass * 1e-3) / 1e12 / fp32_peak, "peak_source": fp32_src}}
    wf = read_profile_value("k_vis_fast_batch_c5_8192", "shared_wavefronts_per_launch")
    if wf is not None:
        binding["shared_memory"] = {"achieved_wavefronts_per_s": wf / (t_pass * 1e-3), "peak": peak_wf,
                                    "frac": wf / (t_pass * 1e-3) / peak_wf, "per_launch": wf,
                                    "peak_source": wf_src}

    # ---- e2e through the reference-facing C ABI with pinned host buffers -----------
    e2e = None
    if c5.plans:
        gk_h, dk_h, sup_h = c5.gk.cpu().numpy(), c5.dk.cpu().numpy(), c5.sup_h
        cfg = S.make_config(G, base.cfg.uv_scale, base.cfg.w_scale, OS)

        def pinned(a):
            t = torch.empty(a.shape, dtype=torch.float32).pin_memory()
            t.numpy()[...] = a
            return t

        uvw_p = [pinned(h[0]) for h in c5.host]
        meas_p = [pinned(h[1]) for h in c5.host]
        mgrid_p = pinned(c5.model.cpu().numpy())
        nmax = max(c5.counts)
        pred_p = torch.empty((nmax, 2), dtype=torch.float32).pin_memory()
        delta_p = torch.empty((nmax, 2), dtype=torch.float32).pin_memory()
        grid_p = torch.empty((G * G, 2), dtype=torch.float32).pin_memory()
        A.set_degrid_mode(S.SDP_DEGRID_CONV)

        def e2e_step():
            for k in range(len(c5.plans)):
                n = c5.counts[k]
                u, m = uvw_p[k].numpy(), meas_p[k].numpy()
                p, d = pred_p.numpy()[:n], delta_p.numpy()[:n]
                A.std_degridding(cfg, G, OS, dk_h, sup_h, mgrid_p.numpy(), u, out=p)
                A.subtract_finegrid(m, p, out=d)
                A.std_gridding(cfg, G, OS, gk_h, sup_h, u, d, out=grid_p.numpy())

        e2e_step()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        t_e2e = (time.perf_counter() - t0) / args.e2e_steps
        A.set_degrid_mode(S.SDP_DEGRID_NEAREST)
        ksz = gk_h.nbytes + sup_h.nbytes
        h2d = sum((n * 12 + G * G * 8 + ksz) + 2 * n * 8 + (ksz + n * 12 + n * 8) for n in c5.counts)
        d2h = sum(n * 8 + n * 8 + G * G * 8 for n in c5.counts)
        e2e = (t_e2e, h2d, d2h)
        del uvw_p, meas_p, mgrid_p, pred_p, delta_p, grid_p
    else:
        t_e2e, h2d, d2h = 0.0, 0, 0
        if world > 1:
            dist.barrier()
    t_e2e = channels.max_over_ranks(e2e[0] if e2e else 0.0, device=dev)
    h2d = e2e[1] if e2e else 0
    d2h = e2e[2] if e2e else 0

    # ---- CPU baseline (rank 0, N = 1): the reference on a sample of the workload ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ref = ReferencePass(base, args.cpu_sample, cpu_threads())
        ref.run(20_000)
        t_cpu = ref.run()
        cpu = {"value": C5_CHANNELS * ref.sample / t_cpu, "unit": UNIT, "cores": ref.threads, "kind": ref.kind,
               "sample": ref.describe()}
        del ref

    # ---- further blocks (one GPU only) ---------------------------------------------------
    extras = {}
    if args.peaks:
        extras["peaks_measured"] = args.peaks
    if world == 1:
        if not args.no_major_cycle and not args.no_extras:
            extras["c5_major_cycle_8192"] = c5_major_cycle_block(S, D, dev, c5)
    c5.close()
    c5 = None
    del flush
    torch.cuda.empty_cache()
    if world == 1 and not args.no_c4:
        extras["c5_learned"] = c5_learned_block(S, D, dev, base, tune, skies=args.c5_skies)
    if world == 1:
        if not args.no_c2:
            extras["c2_2048"] = c2_block(S, D, dev, args)
        if not args.no_c3:
            extras["c3_batched"] = c3_block(S, D, dev)
        if not args.no_c4:
            extras["c4_learned"] = c4_learned_block(S, D, dev, args.c4_skies)
        if not args.no_extras:
            extras["fft_2048"] = fft_block(S, D, dev)
            extras["gain_calibration"] = calibration_block(S, D, dev, not args.no_cpu_baseline)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": t_step, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": c5_config_name(total_vis) + ("" if nch == C5_CHANNELS else
                                                            f" (first {nch} of the 16 channels)"),
                   "channels_per_rank": [len(o) for o in channels.assign_channels(counts_all, world)],
                   "degrid": "convolutional (normalised, degridgrid.c:147-191)",
                   "measured": "exact DFT of 1000 points + 50 Gaussians (sdp_dft_gauss) + 0.1 mJy noise",
                   "l2": "inputs of several GB (larger than L2); L2 also flushed between timed steps (256 MB write)",
                   "exchange": "none at N = 1; N > 1: per-rank channel sum + NCCL all-reduce of the 8192^2 "
                               "continuum residual grid each step" if world > 1 else "none (N = 1)",
                   "work_items": n_items, "plan_shape": tune, "setup_s": setup_s},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_source": peak_src,
                     "kernel": "sdp_visbatch_cycle: residual-grid clears + k_vis_fast_batch<float, %s warps>"
                               % ((tune or {}).get("warps") or "auto"),
                     "algorithmic_bytes_per_launch": alg_bytes, "fp32_flops_per_launch": alg_flops,
                     "ms_per_launch": t_pass},
        "roofline_binding": binding,
        "e2e": {"value": total_vis / t_e2e if t_e2e > 0 else None, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "path": "per channel std_degridding + subtract_from_measurements_finegrid + std_gridding "
                        "(host buffers, pinned), all 16 channels per step"},
        "gpu_launches": args.steps * (2 if world > 1 else 1),
        "clocks": csum,
    }
    line.update(extras)
    if cpu is not None:
        line["cpu_baseline"] = cpu
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
