"""Learned CLEAN proposals: training data, training, and the learned major
cycle with Hogbom as both the fallback and the judge.

No counterpart in the reference (its deconvolution is the Hogbom CLEAN of
deconvolution_run.c:197-311 in the DFT / FFT pipelines).  Everything that
computes runs as libsdp_b200 kernels on the device; torch owns the memory.

* ``Imaging``: one channel of an array imaged at G x G through the library:
  visibilities -> w-projection gridding -> FFT -> taper correction, scaled to
  flux units by the PSF peak, so a point of flux I images with peak ~I.
* ``SkySampler``: seeded random skies of points and circular Gaussians.
* ``make_pair``: the dirty image of a sky (DFT predict of its components -
  the exact form of degridding the sky - plus noise, gridded back) and the
  sky rendered on the pixel grid.
* ``train``: the U-Net trained on random crops of such pairs with the
  blurred squared error and Adam, all on the device.
* ``Deconvolver``: the major cycle, plain (Hogbom components, DFT predict)
  or learned: the network proposes up to max_components components from the
  residual; their visibilities (DFT of pixel components, phase reduced
  exactly in fixed point) are gridded to an image, the least-squares
  step alpha = <R, I>/<I, I> scales them, and the candidate residual is
  recomputed from the visibilities (measured - model - alpha x proposal),
  i.e. one exact degrid/grid major cycle.  The proposal is kept only when
  the residual RMS (FP64) falls; otherwise the cycle runs Hogbom.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

import sdp_b200 as S
import synth

WEIGHTS = Path(__file__).resolve().parent / "weights" / "unet_c4.npz"
# network trained for the 512-antenna 40 km array's 16-channel continuum PSF
WEIGHTS_C5 = Path(__file__).resolve().parent / "weights" / "unet_c5.npz"
CROP_MARGIN = 64  # pixels of image kept around the proposal window for the network


def _torch():
    import torch
    return torch


@dataclass
class ArrayLayout:
    """uvw (wavelengths) of one channel and the imaging geometry."""
    uvw: np.ndarray
    grid_size: int
    cell: float
    max_w: float

    @property
    def uv_scale(self) -> float:
        return self.cell * self.grid_size


def spiral_layout(grid_size: int = 1024, n_ant: int = 256, radius_m: float = 5000.0, n_time: int = 120,
                  freq_hz: float = 140e6, seed: int = 2) -> ArrayLayout:
    """The 256-antenna 10 km log spiral, 120 time steps over +-1 h (32,640 x
    120 = 3,916,800 visibilities), cell chosen so the longest baseline
    reaches 0.9 of the half grid."""
    rng = np.random.default_rng(seed)
    enu = synth.layout_log_spiral(n_ant, radius_m, rng)
    uvw = synth.uvw_tracks(enu, -27.0, -30.0, np.linspace(-1.0, 1.0, n_time), freq_hz)
    uv_max = float(np.max(np.abs(uvw[:, :2])))
    return ArrayLayout(uvw.astype(np.float32), grid_size, 0.45 / uv_max, float(np.max(np.abs(uvw[:, 2]))) * 1.0001)


def c5_channels(time_stride: int = 1, n_channels: int = 16, f_lo: float = 100e6, f_hi: float = 200e6,
                seed: int = 5):
    """The 512-antenna, 40 km log spiral (seed 5), 200 time steps over +-1 h,
    n_channels evenly spaced over f_lo-f_hi: (per-channel uvw in wavelengths,
    cell, max_w), the cell chosen so the longest baseline at f_hi reaches 0.9
    of the half grid (uv_max * cell * G = 0.45 G, for any G), max_w the
    largest |w| at f_hi.  Every time_stride-th time step is kept (1: all)."""
    rng = np.random.default_rng(seed)
    enu = synth.layout_log_spiral(512, 20000.0, rng)
    top = synth.uvw_tracks(enu, -27.0, -30.0, np.linspace(-1.0, 1.0, 200), f_hi)
    uv_max = float(np.max(np.abs(top[:, :2])))
    cell = 0.45 / uv_max
    max_w = float(np.max(np.abs(top[:, 2]))) * 1.0001
    nbl = top.shape[0] // 200
    sub = top.reshape(200, nbl, 3)[::time_stride].reshape(-1, 3)
    freqs = [f_lo + (f_hi - f_lo) * c / (n_channels - 1) for c in range(n_channels)]
    return [np.ascontiguousarray((sub * (f / f_hi)).astype(np.float32)) for f in freqs], cell, max_w


class Imaging:
    """Gridding + FFT imaging of one channel, in flux units (dirty image / PSF peak)."""

    def __init__(self, D: S.Device, layout: ArrayLayout, num_planes: int = 17, half_support: int = 4,
                 oversampling: int = 16):
        torch = _torch()
        self.D = D
        self.layout = layout
        G = self.G = layout.grid_size
        dev = self.dev = torch.device("cuda", torch.cuda.current_device())
        fov = layout.cell * G
        w_scale = (num_planes - 1) ** 2 / layout.max_w
        self.gk, self.dk, self.sup = D.wkernels_generate([half_support] * num_planes, oversampling, layout.max_w, fov)
        sup_h = self.sup.cpu().numpy()
        self.wk = S.Device.wkernels(self.gk, self.sup, sup_h)
        uvw_raw = torch.from_numpy(layout.uvw).to(dev)
        self.uvw_raw = uvw_raw
        self.uvw = torch.empty_like(uvw_raw)
        D.correct_to_finegrid(G, oversampling, layout.uv_scale, uvw_raw, self.uvw)
        self.n = int(self.uvw.shape[0])
        self.plan = D.plan(G, oversampling, layout.uv_scale, w_scale, self.uvw, self.wk, self.wk,
                           keep=(self.uvw, self.gk, self.dk, self.sup))
        self.prol = torch.empty(G // 2 + 1, dtype=torch.float32, device=dev)
        D.prolate_table(G, self.prol)
        self.psf = torch.empty(G * G, dtype=torch.float32, device=dev)
        self.psf_max = D.psf_generate(self.plan, self.prol, self.psf)
        self.grid = torch.empty((G * G, 2), dtype=torch.float32, device=dev)
        self.work = torch.empty_like(self.grid)

    def image(self, vis, out):
        """out (G^2) = image of vis in flux units."""
        self.plan.grid(vis, self.grid)
        self.D.grid_to_image(self.G, self.grid, self.prol, self.work, out)
        self.D.scale(out, 1.0 / self.psf_max)

    def close(self):
        self.plan.close()


class ContinuumImaging:
    """Several channels imaged into one continuum (multi-frequency) image,
    with the interface Deconvolver uses: the visibilities of all channels
    are one array (channel-major), so a DFT predict or a sky's visibilities
    is one launch over every channel (uvw in wavelengths carry the
    frequency); image() grids each channel with its own plan into one
    continuum grid (accumulating), then FFT + taper, in flux units of the
    continuum PSF's peak.  channel_uvw: raw uvw (wavelengths) per channel;
    the geometry (cell, max_w) is shared.  Kernels are generated on the GPU."""

    def __init__(self, D: S.Device, channel_uvw, grid_size: int, cell: float, max_w: float, num_planes: int = 64,
                 half_support: int = 4, oversampling: int = 16, options: "S.PlanOptions | None" = None):
        torch = _torch()
        self.D = D
        G = self.G = grid_size
        dev = self.dev = torch.device("cuda", torch.cuda.current_device())
        self.layout = ArrayLayout(np.zeros((0, 3), np.float32), G, cell, max_w)
        fov = cell * G
        us, ws = cell * G, (num_planes - 1) ** 2 / max_w
        self.gk, self.dk, self.sup = D.wkernels_generate([half_support] * num_planes, oversampling, max_w, fov)
        sup_h = self.sup.cpu().numpy()
        self.wk = S.Device.wkernels(self.gk, self.sup, sup_h)
        counts = [int(u.shape[0]) for u in channel_uvw]
        self.offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        self.n = int(self.offsets[-1])
        self.uvw_raw = torch.empty((self.n, 3), dtype=torch.float32, device=dev)
        self.plans = []
        snapped = torch.empty((max(counts), 3), dtype=torch.float32, device=dev)
        for c, u in enumerate(channel_uvw):
            a, b = int(self.offsets[c]), int(self.offsets[c + 1])
            raw = self.uvw_raw[a:b]
            raw.copy_(torch.as_tensor(u, device=dev))
            sn = snapped[: b - a]
            D.correct_to_finegrid(G, oversampling, us, raw, sn)
            self.plans.append(D.plan(G, oversampling, us, ws, sn, self.wk, self.wk,
                                     keep=(self.gk, self.dk, self.sup), options=options))
        torch.cuda.synchronize()
        del snapped
        self.prol = torch.empty(G // 2 + 1, dtype=torch.float32, device=dev)
        D.prolate_table(G, self.prol)
        self.grid = torch.empty((G * G, 2), dtype=torch.float32, device=dev)
        self.work = torch.empty_like(self.grid)
        # continuum PSF: unit visibilities of every channel, imaged; peak 1
        ones = torch.zeros((max(counts), 2), dtype=torch.float32, device=dev)
        ones[:, 0] = 1.0
        for c, pl in enumerate(self.plans):
            pl.grid(ones[: int(self.offsets[c + 1] - self.offsets[c])], self.grid, accumulate=c > 0)
        del ones
        self.psf = torch.empty(G * G, dtype=torch.float32, device=dev)
        D.grid_to_image(G, self.grid, self.prol, self.work, self.psf)
        self.psf_max = float(self.psf.max().item())
        self.psf /= self.psf_max

    def image(self, vis, out):
        """out (G^2) = continuum image of vis (all channels) in flux units."""
        for c, pl in enumerate(self.plans):
            pl.grid(vis[int(self.offsets[c]):int(self.offsets[c + 1])], self.grid, accumulate=c > 0)
        self.D.grid_to_image(self.G, self.grid, self.prol, self.work, out)
        self.D.scale(out, 1.0 / self.psf_max)

    def close(self):
        for pl in self.plans:
            pl.close()
        self.plans = []


class SkySampler:
    """Seeded skies: 10-500 points (log-uniform 1e-3-1 Jy) and 0-20 circular
    Gaussians (FWHM 2-10 px, log-uniform 1e-2-1 Jy), centred on pixels in
    the central half of the field."""

    def __init__(self, grid_size: int, cell: float, seed: int, points=(10, 500), gaussians=(0, 20),
                 point_flux=(1e-3, 1.0), gauss_flux=(1e-2, 1.0), fwhm_px=(2.0, 10.0)):
        self.G, self.cell = grid_size, cell
        self.rng = np.random.default_rng(seed)
        self.points, self.gaussians = points, gaussians
        self.point_flux, self.gauss_flux, self.fwhm_px = point_flux, gauss_flux, fwhm_px

    def _loguniform(self, lo_hi, n):
        lo, hi = lo_hi
        return np.exp(self.rng.uniform(math.log(lo), math.log(hi), n))

    def sample(self) -> np.ndarray:
        """(n, 4) float32 (l, m, flux, sigma), sigma in direction cosines (0: point)."""
        G, r = self.G, self.rng
        n_p = int(r.integers(self.points[0], self.points[1] + 1))
        n_g = int(r.integers(self.gaussians[0], self.gaussians[1] + 1))
        xy = r.integers(G // 4, 3 * G // 4, size=(n_p + n_g, 2))
        out = np.zeros((n_p + n_g, 4), np.float64)
        out[:, 0] = (xy[:, 0] - G // 2) * self.cell
        out[:, 1] = (xy[:, 1] - G // 2) * self.cell
        out[:n_p, 2] = self._loguniform(self.point_flux, n_p)
        out[n_p:, 2] = self._loguniform(self.gauss_flux, n_g)
        fwhm = r.uniform(self.fwhm_px[0], self.fwhm_px[1], n_g)
        out[n_p:, 3] = fwhm / (2.0 * math.sqrt(2.0 * math.log(2.0))) * self.cell
        return out.astype(np.float32)


def measured_vis(img: Imaging, comps_dev, vis_out, noise_sigma: float, gen):
    """Visibilities of a sky (exact DFT of points and Gaussians) plus complex
    Gaussian noise of the given sigma per component."""
    torch = _torch()
    img.D.dft_gauss(comps_dev, img.uvw_raw, vis_out)
    if noise_sigma > 0:
        vis_out.add_(torch.randn(vis_out.shape, device=vis_out.device, generator=gen), alpha=noise_sigma)


def make_pair(img: Imaging, comps_dev, vis, dirty, sky, noise_sigma: float, gen):
    """dirty (G^2): the sky's visibilities gridded and imaged; sky (G^2): the
    components rendered on the pixel grid."""
    measured_vis(img, comps_dev, vis, noise_sigma, gen)
    img.image(vis, dirty)
    sky.zero_()
    img.D.sky_render(img.G, img.layout.cell, comps_dev, sky)


# ---------------------------------------------------------------------------
# Training
# ---------------------------------------------------------------------------
IN_CHANNELS = 3  # residual / s, signed square root of it, PSF


def init_params(net: S.UNet, in_channels: int, rng: np.random.Generator) -> np.ndarray:
    """He-normal 3x3 weights (fan-in: 9 x the real input channels), zero on
    the padded input channels, zero biases; head weights N(0, 0.01 / base)
    so the first outputs are near zero."""
    p = np.zeros(net.num_params, np.float32)
    for k in range(14):
        cin, cout, wo, bo = net.layer(k)
        real_in = in_channels if k == 0 else cin
        w = rng.standard_normal((9, cout, cin)) * math.sqrt(2.0 / (9 * real_in))
        if k == 0:
            w[:, :, in_channels:] = 0.0
        p[wo:bo] = w.astype(np.float32).reshape(-1)
    cin, _, wo, bo = net.layer(14)
    p[wo:bo] = (0.1 * rng.standard_normal(cin) / math.sqrt(cin)).astype(np.float32)
    return p


@dataclass
class TrainConfig:
    skies: int = 20000
    skies_per_step: int = 4
    crops_per_sky: int = 4
    crop: int = 256
    lr: float = 6e-4
    lr_final: float = 2e-5
    warmup: int = 100
    noise_sigma: float = 1e-4
    seed: int = 1234
    log_every: int = 100
    # residual phase: from residual_start (fraction of the steps) on, each sky
    # is with probability residual_fraction replaced by the residual the
    # current network's verified proposal leaves (target: the sky minus the
    # accepted model), so the network also learns the later cycles' inputs
    residual_start: float = 0.4
    residual_fraction: float = 0.5
    refresh_every: int = 50
    max_components: int = 1024
    rel_threshold: float = 0.05
    alpha_max: float = 2.0


@dataclass
class TrainLog:
    steps: list = field(default_factory=list)
    loss: list = field(default_factory=list)
    seconds: float = 0.0
    skies: int = 0
    residual_skies: int = 0


class _Proposer:
    """Inference copy of the network at G x G and the buffers of one
    verified proposal (used by training to make residual examples)."""

    def __init__(self, img: Imaging, cfg: TrainConfig):
        torch = _torch()
        G, dev = img.G, img.dev
        self.img, self.cfg = img, cfg
        self.net = S.UNet(img.D.lib, IN_CHANNELS, 1, G, G, training=False)
        f32 = dict(dtype=torch.float32, device=dev)
        self.planes = torch.empty((1, IN_CHANNELS, G, G), **f32)
        self.out = torch.empty((1, G, G), **f32)
        self.scale = torch.empty(1, **f32)
        self.comps = torch.empty((cfg.max_components, 4), **f32)
        self.count = torch.zeros(1, dtype=torch.int32, device=dev)
        self.delta = torch.empty(G * G, **f32)
        self.vis = torch.empty((img.n, 2), **f32)
        self.pimg = torch.empty(G * G, **f32)
        self.dots = torch.empty(2, dtype=torch.float64, device=dev)
        self.ws = img.D.select_workspace()

    def residual(self, dirty, sky) -> bool:
        """dirty -= alpha I(proposal), sky -= alpha proposal; False when the
        network proposes nothing."""
        D, G, cfg = self.img.D, self.img.G, self.cfg
        D.unet_input_planes(G, dirty, self.img.psf, self.planes, self.scale)
        self.net.forward(self.planes, self.out)
        D.select_components(G, self.img.layout.cell, self.out, self.scale, cfg.rel_threshold, cfg.max_components,
                            self.comps, self.count, self.delta, self.ws, signed=True)
        n = int(self.count.item())
        if n == 0:
            return False
        D.dft_pixels(self.comps[:n], self.img.layout.cell, self.img.uvw_raw, self.vis)
        self.img.image(self.vis, self.pimg)
        D.dots(dirty, self.pimg, self.dots)
        D.axpy_ratio(self.dots, cfg.alpha_max, self.pimg, dirty, sign=-1.0)
        D.axpy_ratio(self.dots, cfg.alpha_max, self.delta, sky, sign=-1.0)
        return True

    def close(self):
        self.net.close()


def train(img: Imaging, cfg: TrainConfig, params: np.ndarray | None = None, verbose: bool = True):
    """Trains the U-Net from He initialisation (or params) on cfg.skies
    random skies, each giving crops_per_sky random crops.  Returns
    (params, TrainLog)."""
    torch = _torch()
    D, G, dev = img.D, img.G, img.dev
    B = cfg.skies_per_step * cfg.crops_per_sky
    cr = cfg.crop
    net = S.UNet(D.lib, IN_CHANNELS, B, cr, cr, training=True)
    rng = np.random.default_rng(cfg.seed)
    net.set_params(params if params is not None else init_params(net, IN_CHANNELS, rng))
    sampler = SkySampler(G, img.layout.cell, cfg.seed + 1)
    gen = torch.Generator(device=dev).manual_seed(cfg.seed + 2)
    vis = torch.empty((img.n, 2), dtype=torch.float32, device=dev)
    dirty = torch.empty(G * G, dtype=torch.float32, device=dev)
    sky = torch.empty(G * G, dtype=torch.float32, device=dev)
    planes = torch.empty((IN_CHANNELS, G, G), dtype=torch.float32, device=dev)
    s = torch.empty(1, dtype=torch.float32, device=dev)
    xb = torch.empty((B, IN_CHANNELS, cr, cr), dtype=torch.float32, device=dev)
    tb = torch.empty((B, cr, cr), dtype=torch.float32, device=dev)
    out = torch.empty_like(tb)
    grad = torch.empty_like(tb)
    scratch = torch.empty(2 * tb.numel(), dtype=torch.float32, device=dev)
    loss = torch.zeros(1, dtype=torch.float64, device=dev)
    psf2 = img.psf.view(G, G)
    pc = psf2[G // 2 - cr // 2:G // 2 + cr // 2, G // 2 - cr // 2:G // 2 + cr // 2]
    steps = max(1, cfg.skies // cfg.skies_per_step)
    res_from = int(cfg.residual_start * steps)
    proposer = _Proposer(img, cfg) if cfg.residual_fraction > 0 and res_from < steps else None
    log = TrainLog()
    lo, hi = G // 4 - cr // 4, 3 * G // 4 - 3 * cr // 4
    t0 = time.perf_counter()
    for step in range(steps):
        if proposer is not None and step >= res_from and (step - res_from) % cfg.refresh_every == 0:
            proposer.net.set_params(net.get_params())
        b = 0
        for _ in range(cfg.skies_per_step):
            comps = torch.from_numpy(sampler.sample()).to(dev)
            make_pair(img, comps, vis, dirty, sky, cfg.noise_sigma, gen)
            if proposer is not None and step >= res_from and rng.random() < cfg.residual_fraction:
                log.residual_skies += int(proposer.residual(dirty, sky))
            D.unet_input_planes(G, dirty, img.psf, planes, s)
            sky.div_(s)
            sk = sky.view(G, G)
            for _ in range(cfg.crops_per_sky):
                y0, x0 = (int(v) for v in rng.integers(lo, hi + 1, 2))
                xb[b, :2].copy_(planes[:2, y0:y0 + cr, x0:x0 + cr])
                xb[b, 2].copy_(pc)
                tb[b].copy_(sk[y0:y0 + cr, x0:x0 + cr])
                b += 1
        if step < cfg.warmup:
            lr = cfg.lr * (step + 1) / cfg.warmup
        else:
            f = (step - cfg.warmup) / max(1, steps - cfg.warmup)
            lr = cfg.lr_final + 0.5 * (cfg.lr - cfg.lr_final) * (1.0 + math.cos(math.pi * f))
        net.forward(xb, out)
        D.blur_mse(out, tb, scratch, grad, loss)
        net.zero_grads()
        net.backward(grad)
        net.adam_step(lr)
        if (step + 1) % cfg.log_every == 0 or step == steps - 1:
            torch.cuda.synchronize()
            lv = float(loss.item())
            log.steps.append(step + 1)
            log.loss.append(lv)
            if verbose:
                print(f"step {step + 1}/{steps} loss {lv:.3e} lr {lr:.2e} "
                      f"{time.perf_counter() - t0:.1f}s", flush=True)
    torch.cuda.synchronize()
    log.seconds = time.perf_counter() - t0
    log.skies = steps * cfg.skies_per_step
    p = net.get_params()
    net.close()
    if proposer is not None:
        proposer.close()
    return p, log


def save_weights(params: np.ndarray, path: Path = WEIGHTS) -> None:
    """Stores the weights as their BF16 bit patterns (the network computes
    with the BF16 rounding of the weights; the biases are rounded too)."""
    bits = np.asarray(params, np.float32).view(np.uint32)
    bf = ((bits + 0x7FFF + ((bits >> 16) & 1)) >> 16).astype(np.uint16)
    path.parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(path, bf16=bf)


def load_weights(path: Path = WEIGHTS) -> np.ndarray:
    with np.load(path) as z:
        return (z["bf16"].astype(np.uint32) << 16).view(np.float32)


# ---------------------------------------------------------------------------
# Major cycle: plain Hogbom or learned proposals
# ---------------------------------------------------------------------------
@dataclass
class CycleRecord:
    kind: str        # "hogbom" or "learned"
    rms: float       # residual RMS after the cycle (FP64)
    seconds: float   # wall time since the start (device synchronised)
    components: int
    alpha: float = 0.0
    rejected: bool = False


class Deconvolver:
    """Major cycles on one channel.  The residual image of a model is the
    image of (measured - model visibilities); the model's visibilities are
    the exact DFT of its components.

    plain: each cycle runs num_minor Hogbom minor cycles (loop gain) on the
    residual, the new components' visibilities are added to the model and
    the residual is imaged again from the visibilities.
    learned: each cycle first asks the network for a proposal: up to
    max_components components (largest |value| of its output), their
    visibilities (exact DFT) imaged through the gridder (I), the
    least-squares step alpha = <R, I> / <I, I> (clipped to [0, alpha_max]),
    and the candidate residual R - alpha I, which by the linearity of
    gridding and imaging is the image of measured - (model + alpha x
    proposal) visibilities.  The proposal is kept when the residual RMS
    (FP64) falls by more than min_gain (relative); otherwise the cycle runs
    Hogbom, the network is asked again in the next cycle, and after give_up
    rejections it is not asked again.
    Proposals come from the central window (fraction `window` of each axis):
    the outer band of the image holds the taper correction's amplified
    imaging errors (w-term truncation, aliasing), which the network, trained
    on 1024^2 images, reads as sources at 2048^2."""

    def __init__(self, img: Imaging, params: np.ndarray | None, num_minor: int = 200, loop_gain: float = 0.1,
                 max_components: int = 1024, rel_threshold: float = 0.05, alpha_max: float = 2.0,
                 min_gain: float = 0.05, give_up: int = 3, noise_factor: float = 1.5,
                 weak_source_percent: float = 0.0002, signed: bool = True, window: float = 0.75,
                 crop: bool = True):
        torch = _torch()
        self.img, self.D = img, img.D
        G, dev, n = img.G, img.dev, img.n
        self.num_minor, self.max_components = num_minor, max_components
        self.rel_threshold, self.alpha_max, self.min_gain, self.give_up = rel_threshold, alpha_max, min_gain, give_up
        self.signed = signed
        self.border = int(round(G * (1.0 - window) / 2.0))
        # the network runs on the centred crop that holds the proposal window
        # plus a margin wider than its receptive field (radius < 64 pixels:
        # 2 convolutions per level, 2 x 2 pooling, 4 levels), offset a
        # multiple of 16 so the pooling levels line up with the full image's;
        # its output inside the window is then the full image's
        off = max(0, (self.border - CROP_MARGIN) // 16 * 16) if crop else 0
        self.crop_off, self.W = off, G - 2 * off
        self.params = S.CleanParams(G, num_minor, num_minor, loop_gain, noise_factor, weak_source_percent, 1.0,
                                    img.layout.cell)
        self.net = None
        if params is not None:
            self.net = S.UNet(img.D.lib, IN_CHANNELS, 1, self.W, self.W, training=False)
            self.net.set_params(params)
        f32 = dict(dtype=torch.float32, device=dev)
        self.model_vis = torch.zeros((n, 2), **f32)
        self.prop_vis = torch.empty((n, 2), **f32)
        self.delta_vis = torch.empty((n, 2), **f32)
        self.residual = torch.empty(G * G, **f32)
        self.cand = torch.empty(G * G, **f32)
        self.prop_img = torch.empty(G * G, **f32)
        self.clean_img = torch.empty(G * G, **f32)
        self.model_img = torch.zeros(G * G, **f32)
        self.planes = torch.empty((1, IN_CHANNELS, self.W, self.W), **f32)
        self.out = torch.empty((1, self.W, self.W), **f32)
        self.scale = torch.empty(1, **f32)
        self.comps = torch.empty((max_components, 4), **f32)
        self.count = torch.zeros(1, dtype=torch.int32, device=dev)
        self.sources = torch.empty((num_minor, 3), **f32)
        self.nsrc = torch.zeros(1, dtype=torch.int32, device=dev)
        self.dots = torch.empty(2, dtype=torch.float64, device=dev)
        self.alpha = torch.empty(1, **f32)
        self.sel_ws = img.D.select_workspace()
        self.clean_ws = torch.empty(img.D.hogbom_workspace_bytes(G), dtype=torch.uint8, device=dev)

    def close(self):
        if self.net is not None:
            self.net.close()
            self.net = None

    def _residual(self, measured):
        self.D.subtract_vis(measured, self.model_vis, self.delta_vis)
        self.img.image(self.delta_vis, self.residual)
        return self.D.image_rms(self.img.G, self.residual)

    def _hogbom(self, measured) -> tuple[float, int]:
        D = self.D
        self.clean_img.copy_(self.residual)
        D.hogbom(self.params, self.clean_img, self.img.psf, self.model_img, self.sources, self.nsrc, self.clean_ws)
        n = int(self.nsrc.item())
        if n > 0:
            D.dft_pixels(self.sources[:n], self.img.layout.cell, self.img.uvw_raw, self.model_vis, accumulate=True)
        return self._residual(measured), n

    def _select(self) -> int:
        """The network's proposal for the current residual: components in
        self.comps, returns their number."""
        D, G, W = self.D, self.img.G, self.W
        D.unet_input_planes_window(G, W, self.residual, self.img.psf, self.planes, self.scale)
        self.net.forward(self.planes, self.out)
        D.zero_border(W, self.border - self.crop_off, self.out)
        # a centred crop keeps (x - W/2) cell = (x + off - G/2) cell
        D.select_components(W, self.img.layout.cell, self.out, self.scale, self.rel_threshold,
                            self.max_components, self.comps, self.count, None, self.sel_ws, signed=self.signed)
        return int(self.count.item())

    def _propose(self, rms) -> tuple[bool, float, float, int]:
        D, G = self.D, self.img.G
        n = self._select()
        if n == 0:
            return False, rms, 0.0, 0
        D.dft_pixels(self.comps[:n], self.img.layout.cell, self.img.uvw_raw, self.prop_vis)
        self.img.image(self.prop_vis, self.prop_img)
        D.dots(self.residual, self.prop_img, self.dots)
        self.cand.copy_(self.residual)
        D.axpy_ratio(self.dots, self.alpha_max, self.prop_img, self.cand, self.alpha, sign=-1.0)
        new = D.image_rms(G, self.cand)
        a = float(self.alpha.item())
        if new < rms * (1.0 - self.min_gain) and a > 0.0:
            D.axpy_ratio(self.dots, self.alpha_max, self.prop_vis, self.model_vis, sign=1.0)
            self.residual, self.cand = self.cand, self.residual
            return True, new, a, n
        return False, rms, a, n

    def exact_residual(self, measured):
        """(tracked residual image, residual imaged afresh from measured -
        model visibilities, RMS of the latter) for the state a run left."""
        tracked = self.residual.clone()
        rms = self._residual(measured)
        return tracked, self.residual.clone(), rms

    def run(self, measured, max_cycles: int, learned: bool, target_rms: float | None = None):
        """Runs up to max_cycles major cycles from an empty model (stops early
        once the residual RMS is at or below target_rms).  Returns the
        initial RMS and one CycleRecord per cycle; times are wall-clock with
        the device synchronised, from before the first imaging."""
        torch = _torch()
        self.model_vis.zero_()
        self.model_img.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rms = self._residual(measured)
        rms0 = rms
        recs = []
        rejections = 0
        for _ in range(max_cycles):
            done = False
            if learned and self.net is not None and rejections < self.give_up:
                ok, new, a, n = self._propose(rms)
                if ok:
                    rms = new
                    torch.cuda.synchronize()
                    recs.append(CycleRecord("learned", rms, time.perf_counter() - t0, n, a))
                    done = True
                else:
                    rejections += 1
            if not done:
                rms, n = self._hogbom(measured)
                torch.cuda.synchronize()
                recs.append(CycleRecord("hogbom", rms, time.perf_counter() - t0, n,
                                        rejected=learned and self.net is not None))
            if target_rms is not None and rms <= target_rms:
                break
        return rms0, recs


def time_to_target(recs, target: float):
    """(seconds, cycles) of the first cycle at or below target, or (None, None)."""
    for k, r in enumerate(recs):
        if r.rms <= target:
            return r.seconds, k + 1
    return None, None


def evaluate(img, params: np.ndarray, skies: int, seed: int = 777, plain_cycles: int = 10,
             max_learned_cycles: int = 10, noise_sigma: float = 1e-4, verbose: bool = False, sampler=None, **kw):
    """Held-out skies: the plain pipeline runs plain_cycles Hogbom cycles; its
    final RMS x 1.01 is the target the learned pipeline must reach.  img is
    an Imaging (one channel) or a ContinuumImaging (several channels).
    Returns one dict per sky."""
    torch = _torch()
    dec = Deconvolver(img, params, **kw)
    sampler = sampler or SkySampler(img.G, img.layout.cell, seed)
    gen = torch.Generator(device=img.dev).manual_seed(seed + 1)
    meas = torch.empty((img.n, 2), dtype=torch.float32, device=img.dev)
    rows = []
    for k in range(skies):
        comps = torch.from_numpy(sampler.sample()).to(img.dev)
        measured_vis(img, comps, meas, noise_sigma, gen)
        rms0, plain = dec.run(meas, plain_cycles, learned=False)
        target = plain[-1].rms * 1.01
        _, lrn = dec.run(meas, max_learned_cycles, learned=True, target_rms=target)
        tp, cp = time_to_target(plain, target)
        tl, cl = time_to_target(lrn, target)
        row = dict(sky=k, components=int(comps.shape[0]), rms0=rms0, plain_final=plain[-1].rms, target=target,
                   plain_s=tp, plain_cycles=cp, learned_s=tl, learned_cycles=cl,
                   learned_kinds="".join(r.kind[0] for r in lrn), learned_final=lrn[-1].rms,
                   plain_rms=[r.rms for r in plain], learned_rms=[r.rms for r in lrn],
                   learned_seconds=[r.seconds for r in lrn], plain_seconds=[r.seconds for r in plain])
        rows.append(row)
        if verbose:
            print(row, flush=True)
    dec.close()
    return rows


def main(argv=None) -> int:
    """python learned.py train|eval|forward [--skies N] [--out PATH] [--grid G]

    forward: two forward passes of the committed network on a random
    3 x G x G input (the second timed with CUDA events)."""
    import argparse
    import json
    torch = _torch()
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train", "eval", "forward"])
    ap.add_argument("--skies", type=int, default=20000)
    ap.add_argument("--grid", type=int, default=1024)
    ap.add_argument("--out", type=Path, default=WEIGHTS)
    ap.add_argument("--weights", type=Path, default=WEIGHTS)
    ap.add_argument("--eval-skies", type=int, default=8)
    ap.add_argument("--log", type=Path, default=None)
    ap.add_argument("--config", choices=["c4", "c5"], default="c4",
                    help="c4: one channel of the 10 km array; c5: the 40 km array's 16-channel continuum "
                         "(every 8th time step, imaged at --grid with the 8192^2 image's cell)")
    a = ap.parse_args(argv)
    torch.cuda.init()
    D = S.Device()
    if a.cmd == "forward":
        net = S.UNet(D.lib, IN_CHANNELS, 1, a.grid, a.grid, training=False)
        net.set_params(load_weights(a.weights))
        x = torch.randn((1, IN_CHANNELS, a.grid, a.grid), device="cuda")
        out = torch.empty((1, a.grid, a.grid), device="cuda")
        net.forward(x, out)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        net.forward(x, out)
        e1.record()
        torch.cuda.synchronize()
        net.check()
        print(f"forward {a.grid}^2: {e0.elapsed_time(e1):.3f} ms")
        net.close()
        return 0
    if a.config == "c5":
        chans, cell, max_w = c5_channels(time_stride=8)
        img = ContinuumImaging(D, chans, a.grid, cell, max_w)
        if a.out == WEIGHTS:
            a.out = WEIGHTS_C5
    else:
        img = Imaging(D, spiral_layout(a.grid))
    if a.cmd == "train":
        params, log = train(img, TrainConfig(skies=a.skies))
        save_weights(params, a.out)
        rows = evaluate(img, load_weights(a.out), a.eval_skies, verbose=True)
        if a.log:
            a.log.write_text(json.dumps(dict(steps=log.steps, loss=log.loss, seconds=log.seconds, skies=log.skies,
                                             residual_skies=log.residual_skies, eval=rows), indent=1))
    else:
        rows = evaluate(img, load_weights(a.weights), a.eval_skies, verbose=True)
        if a.log:
            a.log.write_text(json.dumps(dict(eval=rows), indent=1))
    img.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
