"""Generates tests/golden/*.npz from the reference's own actors.

    make -C oracle ref            # compiles the reference sources (needs the reference tree)
    python tests/golden/make_golden.py

Every output stored here was produced by the reference's actor code compiled
unmodified from its sources (oracle/_ref/libref_{f32,f64}.so) on seeded
synthetic inputs; the inputs are stored next to the outputs.  The fixtures pin
the oracle restatement (tests/test_oracle_pins.py) and the CUDA path
(tests/test_gpu_*.py) on machines where the reference tree is absent.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "simsdp-generic-imaging-pipeline_b200"))

import oracle as O  # noqa: E402
import synth  # noqa: E402

OUT = Path(__file__).resolve().parent


def edge_uvw(G: int, uv_scale: float, w_scale: float, n_planes: int, rng) -> np.ndarray:
    """Visibilities at the grid edges and at positions within one float ulp of
    integers (where the reference's float ceil() gives 2hs-1 or 2hs+1 taps)."""
    gc = G // 2
    pts = []
    for gx in (-gc, -gc + 0.5, -gc + 1, gc - 1, gc - 1.5, gc - 0.01, -3.0, 0.0, 3.0, 5.0):
        for gy in (-gc, 0.0, gc - 1, 7.0):
            pts.append((gx, gy))
    for base in (-7, -3, -1, 0, 1, 2, 5, 11):
        for k in range(-3, 4):
            x = np.nextafter(np.float32(base), np.float32(np.inf if k > 0 else -np.inf))
            for _ in range(abs(k) - 1):
                x = np.nextafter(x, np.float32(np.inf if k > 0 else -np.inf))
            if k == 0:
                x = np.float32(base)
            pts.append((float(x), float(base) + 0.25))
            pts.append((float(base) - 0.5, float(x)))
    pts = np.asarray(pts, dtype=np.float64)
    uv = pts / uv_scale
    wmax = ((n_planes - 1) ** 2) / w_scale
    w = rng.uniform(-0.999, 0.999, size=len(pts)) * wmax
    return np.concatenate([uv, w[:, None]], axis=1).astype(np.float32)


def main() -> int:
    if not O.RefLib.available("f32") or not O.RefLib.available("f64"):
        print("compiled reference missing: run make -C oracle ref", file=sys.stderr)
        return 1
    r32, r64 = O.RefLib("f32"), O.RefLib("f64")
    rng = np.random.default_rng(2024)

    # --- W-projection visibility path, FFT pipeline order ---------------------------------
    w = synth.small_workload(seed=11, grid_size=64, n_ant=12, n_time=8, num_planes=4, half_support=2,
                             oversampling=16, n_src=5)
    G, OS = w.cfg.grid_size, w.cfg.oversampling
    cfg = O.make_config(G, w.cfg.uv_scale, w.cfg.w_scale, OS)
    uvw = np.concatenate([w.uvw, edge_uvw(G, w.cfg.uv_scale, w.cfg.w_scale, 4, rng)], axis=0)
    vis = (rng.standard_normal((uvw.shape[0], 2)) * 0.5).astype(np.float32)
    vis[: w.num_vis] = w.vis
    model_grid = rng.standard_normal((G * G, 2)).astype(np.float32)
    fix = dict(grid_size=G, oversampling=OS, uv_scale=w.cfg.uv_scale, w_scale=w.cfg.w_scale,
               uvw=uvw, vis=vis, gkernels=w.gkernels, dkernels=w.dkernels, supports=w.supports,
               model_grid=model_grid)
    ov, ou, n = r32.correct_to_finegrid(cfg, G, OS, uvw, vis)
    fix["ctf_uvw_f32"], fix["ctf_vis_f32"] = ou, ov
    fix["grid_f32"] = r32.std_gridding(cfg, G, OS, w.gkernels, w.supports, ou, vis)
    ov64, ou64, _ = r64.correct_to_finegrid(cfg, G, OS, uvw, vis)
    fix["ctf_uvw_f64"] = ou64
    fix["grid_f64"] = r64.std_gridding(cfg, G, OS, w.gkernels, w.supports, ou64, vis)
    fix["grid_raw_f32"] = r32.std_gridding(cfg, G, OS, w.gkernels, w.supports, uvw, vis)
    fix["degrid_f32"] = r32.std_degridding(cfg, G, OS, w.dkernels, w.supports, model_grid, ou)
    fix["degrid_raw_f32"] = r32.std_degridding(cfg, G, OS, w.dkernels, w.supports, model_grid, uvw)
    fix["subtract_f32"] = r32.subtract_finegrid(vis, fix["degrid_f32"])
    fix["g2g_f32"] = r32.g2g_degridgrid(cfg, G, OS, w.gkernels, w.supports, w.dkernels, w.supports, model_grid, ou)
    fix["g2g_f64"] = r64.g2g_degridgrid(cfg, G, OS, w.gkernels, w.supports, w.dkernels, w.supports, model_grid, ou64)
    fix["gridding_actor_f32"] = r32.gridding_actor(cfg, G, w.gkernels, w.supports, uvw, vis)
    fix["gridding_actor_f64"] = r64.gridding_actor(cfg, G, w.gkernels, w.supports, uvw, vis)
    np.savez_compressed(OUT / "wproj_g64.npz", **fix)

    # --- FFT, shifts, taper ---------------------------------------------------------------
    G = 32
    x = rng.standard_normal((G * G, 2)).astype(np.float32)
    img = rng.standard_normal(G * G).astype(np.float32)
    cfg = O.make_config(G, 1.0, 1.0)
    fix = dict(grid_size=G, x=x, image=img)
    fix["fft_fwd_f32"] = r32.fft(G, x, False)
    fix["fft_inv_f32"] = r32.fft(G, x, True)
    fix["fft_fwd_f64"] = r64.fft(G, x, False)
    fix["fft_inv_f64"] = r64.fft(G, x, True)
    fix["shift_c2c_f32"] = r32.fft_shift_c2c(cfg, G, x)
    fix["shift_c2r_f32"] = r32.fft_shift_c2r(cfg, G, x)
    fix["shift_r2c_f32"] = r32.fft_shift_r2c(cfg, G, img)
    fix["prolate_f32"] = r32.half_prolate_ext(G)
    fix["taper_f32"] = r32.conv_correction(cfg, G, img, fix["prolate_f32"])
    grids = rng.standard_normal((4 * G * G, 2)).astype(np.float32)
    fix["grids4"] = grids
    fix["merge_f32"] = r32.merge_grids(G, grids)
    fix["subimg_f32"] = r32.subtract_image(G, img, img[::-1].copy())
    np.savez_compressed(OUT / "fft_g32.npz", **fix)

    # --- DFT ----------------------------------------------------------------------------------
    w = synth.small_workload(seed=12, grid_size=64, oversampling=16)
    src = np.stack([rng.uniform(-0.05, 0.05, 20), rng.uniform(-0.05, 0.05, 20), rng.uniform(0.01, 1, 20)], 1)
    src = src.astype(np.float32)
    cfg = O.make_config(64, w.cfg.uv_scale, w.cfg.w_scale)
    np.savez_compressed(OUT / "dft.npz", sources=src, uvw=w.uvw, vis_f32=r32.dft(cfg, src, w.uvw),
                        vis_f64=r64.dft(cfg, src, w.uvw))

    # --- Hogbom on a dirty image made by the reference's own imaging actors -------------------
    G = 64
    w = synth.small_workload(seed=13, grid_size=G, n_ant=16, n_time=10, num_planes=4, half_support=2,
                             oversampling=16, n_src=6)
    cfg = O.make_config(G, w.cfg.uv_scale, w.cfg.w_scale, 16, cell_size=w.cfg.cell_size)
    prolate = r32.half_prolate_ext(G)

    def image_of(v):
        g = r32.std_gridding(cfg, G, 16, w.gkernels, w.supports, w.uvw, v)
        g = r32.fft_shift_c2c(cfg, G, g)
        g = r32.fft(G, g, True)
        im = r32.fft_shift_c2r(cfg, G, g)
        return r32.conv_correction(cfg, G, im, prolate)

    dirty = image_of(w.vis)
    psf_full = image_of(np.tile(np.array([[1.0, 0.0]], dtype=np.float32), (w.num_vis, 1)))
    mx, psf = O.Oracle("f32").psf_crop_normalise(G, psf_full)
    cfg.psf_max_value = mx
    n, src, model = r32.hogbom(cfg, G, 100, 200, dirty, psf)
    clean, hd = r32.clean_psf(cfg, G, psf)
    np.savez_compressed(OUT / "hogbom_g64.npz", grid_size=G, dirty=dirty, psf=psf, psf_max=mx,
                        cell_size=w.cfg.cell_size, num_sources=n, sources=src, model=model, clean_psf=clean,
                        halfdims=hd)
    for f in sorted(OUT.glob("*.npz")):
        print(f.name, f.stat().st_size)
    return 0


if __name__ == "__main__":
    sys.exit(main())
