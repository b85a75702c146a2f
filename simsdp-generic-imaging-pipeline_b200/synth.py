"""Seeded synthetic inputs in the reference's array layouts.

The reference pipeline reads GLEAM visibilities, W-projection kernels and a
PSF from CSV files it never generates (param_code/code_fft_1core/src/top.c:
139-237 visibilities, :239-383 kernels, :453-515 PSF).  None of those files
ship with the reference, so every workload here is generated from seeded
random numbers with the shapes the imaging configurations name:

* antenna layouts (uniform disc, log spiral) and Earth-rotation uvw tracks,
  ordered time-major with baselines in the reference's (a, b), a < b order
  (top.c:118-136), in wavelengths (the reference sets frequency_hz = c, so
  its metres are wavelengths, top.c:15, 175);
* point-source skies and their visibilities through the reference's DFT
  formula (dft_run.c:3-48, approximation branch), plus complex noise;
* W-projection gridding/degridding kernels (Cornwell, Golap & Bhatnagar
  2008): the image-domain product of the prolate spheroidal taper used by
  the reference's correction (top.c:412-451) and the paraxial w phase
  screen, oversampled and Fourier transformed.  Tables are stored as the
  reference indexes them: per plane ((hs+1)*OS)^2 complex samples, row
  index |dv|*OS, column index |du|*OS (degridgrid.c:101-112), planes
  concatenated with offsets in supports[:,1] (top.c:256-261).

All arrays are numpy; complex data is returned as interleaved float pairs so
they can be handed to the C ABI as PRECISION2 arrays.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

C_LIGHT = 299792458.0


# ---------------------------------------------------------------------------
# Config mirror (numeric fields of the reference's Config, common.h:187-265,
# with the values config_struct_set_up assigns, top.c:9-68)
# ---------------------------------------------------------------------------
@dataclasses.dataclass
class ImagingConfig:
    grid_size: int
    num_kernels: int = 17
    oversampling: int = 16
    cell_size: float = 8.52211548825356e-06
    max_w: float = 1895.410847844
    loop_gain: float = 0.1
    noise_factor: float = 1.5
    weak_source_percent_img: float = 0.0002
    psf_max_value: float = 0.0

    @property
    def uv_scale(self) -> float:  # top.c:38
        return self.cell_size * self.grid_size

    @property
    def w_scale(self) -> float:  # top.c:36
        return float((self.num_kernels - 1) ** 2) / self.max_w


# ---------------------------------------------------------------------------
# Array layouts and uvw tracks
# ---------------------------------------------------------------------------
def layout_uniform_disc(n_ant: int, radius_m: float, rng: np.random.Generator) -> np.ndarray:
    """East/north antenna positions (metres), uniform in a disc."""
    r = radius_m * np.sqrt(rng.random(n_ant))
    t = 2.0 * np.pi * rng.random(n_ant)
    return np.stack([r * np.cos(t), r * np.sin(t)], axis=1)


def layout_log_spiral(n_ant: int, radius_m: float, rng: np.random.Generator, arms: int = 3,
                      r_min_m: float = 20.0) -> np.ndarray:
    """Three-arm logarithmic spiral with small seeded jitter, radius_m outer radius."""
    per_arm = int(math.ceil(n_ant / arms))
    pos = []
    b = 1.0 / math.tan(math.radians(70.0))  # pitch angle of 70 degrees
    for a in range(arms):
        radii = np.geomspace(r_min_m, radius_m, per_arm)
        theta = np.log(radii / r_min_m) / b + 2.0 * np.pi * a / arms
        x = radii * np.cos(theta)
        y = radii * np.sin(theta)
        jitter = rng.normal(scale=0.01, size=(per_arm, 2)) * radii[:, None]
        pos.append(np.stack([x, y], axis=1) + jitter)
    return np.concatenate(pos, axis=0)[:n_ant]


def baseline_pairs(n_ant: int) -> np.ndarray:
    """(a, b) pairs with a < b in the reference's order (top.c:118-136)."""
    a, b = np.triu_indices(n_ant, k=1)
    return np.stack([a, b], axis=1).astype(np.int32)


def uvw_tracks(enu: np.ndarray, lat_deg: float, dec_deg: float, ha_hours: np.ndarray,
               freq_hz: float) -> np.ndarray:
    """uvw in wavelengths, shape (n_time * n_baseline, 3), time-major.

    Baseline vectors in the local (east, north, up) frame are rotated to the
    equatorial frame and projected onto the (u, v, w) basis of the phase
    centre (Thompson, Moran & Swenson, eq. 4.1-4.2)."""
    lat = math.radians(lat_deg)
    dec = math.radians(dec_deg)
    pairs = baseline_pairs(enu.shape[0])
    e = enu[pairs[:, 1], 0] - enu[pairs[:, 0], 0]
    n = enu[pairs[:, 1], 1] - enu[pairs[:, 0], 1]
    up = np.zeros_like(e)
    X = -math.sin(lat) * n + math.cos(lat) * up
    Y = e
    Z = math.cos(lat) * n + math.sin(lat) * up
    h = np.radians(15.0 * np.asarray(ha_hours, dtype=np.float64))[:, None]
    sh, ch = np.sin(h), np.cos(h)
    u = sh * X + ch * Y
    v = -math.sin(dec) * ch * X + math.sin(dec) * sh * Y + math.cos(dec) * Z
    w = math.cos(dec) * ch * X - math.cos(dec) * sh * Y + math.sin(dec) * Z
    lam = C_LIGHT / freq_hz
    return (np.stack([u, v, w], axis=-1) / lam).reshape(-1, 3)


# ---------------------------------------------------------------------------
# Skies and visibilities
# ---------------------------------------------------------------------------
def point_sky(n_src: int, fov_rad: float, flux_lo: float, flux_hi: float,
              rng: np.random.Generator) -> np.ndarray:
    """(l, m, flux) for n_src points uniform in the central half of the field."""
    half = 0.25 * fov_rad
    lm = rng.uniform(-half, half, size=(n_src, 2))
    flux = np.exp(rng.uniform(math.log(flux_lo), math.log(flux_hi), size=n_src))
    return np.concatenate([lm, flux[:, None]], axis=1)


def dft_visibilities(uvw: np.ndarray, sky: np.ndarray, chunk: int = 1 << 16) -> np.ndarray:
    """Complex128 visibilities of a point sky with the reference's DFT formula
    (dft_run.c:219-230): V = sum I/(1 - r^2/2) exp(-2 pi i (ul + vm - w r^2/2))."""
    l, m, flux = sky[:, 0], sky[:, 1], sky[:, 2]
    term = 0.5 * (l * l + m * m)
    amp = flux / (1.0 - term)
    out = np.empty(uvw.shape[0], dtype=np.complex128)
    for s in range(0, uvw.shape[0], chunk):
        blk = uvw[s:s + chunk]
        theta = 2.0 * np.pi * (np.outer(blk[:, 0], l) + np.outer(blk[:, 1], m) - np.outer(blk[:, 2], term))
        out[s:s + chunk] = (amp[None, :] * np.exp(-1j * theta)).sum(axis=1)
    return out


def add_noise(vis: np.ndarray, sigma: float, rng: np.random.Generator) -> np.ndarray:
    return vis + sigma * (rng.standard_normal(vis.shape) + 1j * rng.standard_normal(vis.shape))


def complex_to_pairs(z: np.ndarray, dtype=np.float32) -> np.ndarray:
    out = np.empty(z.shape + (2,), dtype=dtype)
    out[..., 0] = z.real
    out[..., 1] = z.imag
    return out


# ---------------------------------------------------------------------------
# Prolate spheroidal (Schwab 1984 rational approximation, the form the
# reference evaluates in top.c:412-451) and W-projection kernels
# ---------------------------------------------------------------------------
_P = (0.08203343, -0.3644705, 0.627866, -0.5335581, 0.2312756,
      0.004028559, -0.03697768, 0.1021332, -0.1201436, 0.06412774)
_Q = (1.0, 0.8212018, 0.2078043, 1.0, 0.9599102, 0.2918724)


def prolate(nu: np.ndarray) -> np.ndarray:
    nu = np.abs(np.asarray(nu, dtype=np.float64))
    out = np.zeros_like(nu)
    for part, (lo, hi) in enumerate(((0.0, 0.75), (0.75, 1.0))):
        sel = (nu >= lo) & (nu < hi)
        d = nu[sel] ** 2 - hi * hi
        top = sum(_P[part * 5 + i] * d ** i for i in range(5))
        bot = sum(_Q[part * 3 + i] * d ** i for i in range(3))
        out[sel] = top / bot
    return out


def wproj_kernels(num_planes: int, half_support, oversampling: int, max_w: float, fov_rad: float,
                  image_samples: int = 256):
    """Oversampled W-projection kernel tables.

    Returns (gridding, degridding, supports): two float32 arrays of shape
    (total_samples, 2) and an int32 (num_planes, 2) array of (half support,
    offset).  Plane p holds w = p^2 * max_w / (num_planes-1)^2, the centre of
    the plane index the reference computes, round(sqrt(|w| * w_scale)).

    The taper times the paraxial w screen is separable in (l, m), so each
    plane is the outer product of one 1-D kernel with itself: the 1-D
    kernel is the oversampled Fourier transform of taper(l) exp(-i pi w l^2)
    sampled at image_samples points across the field.  Degridding kernels
    are the complex conjugates.  All planes share the normalisation that
    makes the w = 0 kernel sum to 1 over its taps.
    """
    if np.isscalar(half_support):
        hs_list = [int(half_support)] * num_planes
    else:
        hs_list = [int(h) for h in half_support]
    M = int(image_samples)
    os_ = int(oversampling)
    L = float(fov_rad)
    l = (np.arange(M) - M // 2) * (L / M)
    taper = prolate(2.0 * l / L)
    pad = M * os_
    w_planes = [(p * p) * max_w / float((num_planes - 1) ** 2) if num_planes > 1 else 0.0
                for p in range(num_planes)]
    kernels_1d = []
    for w in w_planes:
        screen = np.zeros(pad, dtype=np.complex128)
        screen[(pad - M) // 2:(pad + M) // 2] = taper * np.exp(-1j * np.pi * w * l * l)
        k = np.fft.fftshift(np.fft.fft(np.fft.ifftshift(screen)))
        kernels_1d.append(k)
    centre = pad // 2
    hs0 = hs_list[0]
    norm = kernels_1d[0][centre + os_ * np.arange(-hs0, hs0 + 1)].sum().real
    tables_g, tables_d, supports = [], [], []
    offset = 0
    for p, k in enumerate(kernels_1d):
        hs = hs_list[p]
        n1 = (hs + 1) * os_
        k1 = k[centre:centre + n1] / norm            # samples at |du| = j / OS
        k2 = np.outer(k1, k1)                        # [|dv|*OS, |du|*OS]
        tables_g.append(complex_to_pairs(k2.reshape(-1)))
        tables_d.append(complex_to_pairs(np.conj(k2).reshape(-1)))
        supports.append((hs, offset))
        offset += n1 * n1
    return (np.concatenate(tables_g, axis=0), np.concatenate(tables_d, axis=0),
            np.asarray(supports, dtype=np.int32))


# ---------------------------------------------------------------------------
# Whole workloads
# ---------------------------------------------------------------------------
@dataclasses.dataclass
class Workload:
    name: str
    cfg: ImagingConfig
    uvw: np.ndarray          # (N, 3) float32 wavelengths, RA flip applied
    vis: np.ndarray          # (N, 2) float32 measured visibilities
    sky: np.ndarray          # (S, 3) float64 (l, m, flux)
    gkernels: np.ndarray     # (K, 2) float32
    dkernels: np.ndarray     # (K, 2) float32
    supports: np.ndarray     # (planes, 2) int32
    half_support: int

    @property
    def num_vis(self) -> int:
        return int(self.uvw.shape[0])


def make_workload(name: str, n_ant: int, radius_m: float, layout: str, n_time: int, grid_size: int,
                  n_src: int, flux_lo: float, flux_hi: float, noise_sigma: float, num_planes: int,
                  half_support: int, oversampling: int = 16, freq_hz: float = 140e6, seed: int = 1,
                  lat_deg: float = -27.0, dec_deg: float = -30.0, ha_span_h: float = 1.0,
                  compute_vis: bool = True, n_vis_cap: int | None = None) -> Workload:
    rng = np.random.default_rng(seed)
    if layout == "disc":
        enu = layout_uniform_disc(n_ant, radius_m, rng)
    else:
        enu = layout_log_spiral(n_ant, radius_m, rng)
    ha = np.linspace(-ha_span_h, ha_span_h, n_time)
    uvw = uvw_tracks(enu, lat_deg, dec_deg, ha, freq_hz)
    if n_vis_cap is not None:
        uvw = uvw[:n_vis_cap]
    uv_max = float(np.max(np.abs(uvw[:, :2])))
    # longest baseline reaches 0.9 of the half grid: uv_max * uv_scale = 0.9 * G/2
    cell = 0.45 / uv_max
    max_w = float(np.max(np.abs(uvw[:, 2]))) * 1.0001
    cfg = ImagingConfig(grid_size=grid_size, num_kernels=num_planes, oversampling=oversampling,
                        cell_size=cell, max_w=max_w)
    fov = cell * grid_size
    sky = point_sky(n_src, fov, flux_lo, flux_hi, rng)
    if compute_vis:
        v = dft_visibilities(uvw, sky)
        v = add_noise(v, noise_sigma, rng)
    else:
        v = (rng.standard_normal(uvw.shape[0]) + 1j * rng.standard_normal(uvw.shape[0])) * 0.1
    g, d, sup = wproj_kernels(num_planes, half_support, oversampling, max_w, fov)
    return Workload(name=name, cfg=cfg, uvw=uvw.astype(np.float32), vis=complex_to_pairs(v),
                    sky=sky, gkernels=g, dkernels=d, supports=sup, half_support=half_support)


def workload_c1(seed: int = 1, compute_vis: bool = True) -> Workload:
    """64 antennas in a 2 km disc, 60 time steps over +-1 h: 2016 x 60 = 120,960
    visibilities at 140 MHz; 512^2 grid, 8 w-planes, support 7 (hs = 3), OS 16;
    50 points of 0.01-1 Jy plus 1 mJy noise."""
    return make_workload("c1_fft_512", 64, 1000.0, "disc", 60, 512, 50, 0.01, 1.0, 1e-3, 8, 3,
                         seed=seed, compute_vis=compute_vis)


def workload_c2(seed: int = 2, compute_vis: bool = False) -> Workload:
    """256 antennas on a 10 km log spiral, 120 time steps: 32,640 x 120 =
    3,916,800 visibilities; 2048^2 grid; 17 w-planes of half support 4 and
    OS 16 (the reference schedule's NUM_KERNELS = 17, TOTAL_KERNEL_SAMPLES =
    108800, code_fft_1core/generated/Core0.c); 200 points of 1e-3-1 Jy."""
    return make_workload("c2_2048", 256, 5000.0, "spiral", 120, 2048, 200, 1e-3, 1.0, 1e-4, 17, 4,
                         seed=seed, compute_vis=compute_vis)


def small_workload(seed: int = 7, grid_size: int = 64, n_ant: int = 12, n_time: int = 8,
                   num_planes: int = 4, half_support: int = 2, oversampling: int = 8,
                   n_src: int = 5) -> Workload:
    """A few hundred visibilities for parity tests that the oracle finishes in
    well under a second."""
    return make_workload(f"small_g{grid_size}", n_ant, 800.0, "disc", n_time, grid_size, n_src, 0.05, 1.0,
                         1e-3, num_planes, half_support, oversampling=oversampling, seed=seed)
