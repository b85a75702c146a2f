"""ORACLE — test infrastructure only.

ctypes front end for two CPU implementations of the reference's imaging
actors:

* ``Oracle(precision)``: this project's C restatement (sdp_oracle.c), built
  into oracle/_build/liboracle_{f32,f64}.so.  It is the checker used by the
  parity tests, by __graft_entry__.smoke() and by bench.py's cpu_baseline leg.
* ``RefLib(precision)``: the reference's own actor sources compiled as they
  are (oracle/Makefile target ``ref`` -> oracle/_ref/libref_*.so).  Used to
  pin the restatement and as the reference arm of bench.py.

Nothing in the product imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"
REFDIR = HERE / "_ref"

_f = C.c_float
_d = C.c_double
_i = C.c_int
_p = C.c_void_p


def build(ref: bool = False) -> None:
    """Compile the restatement (and, when the reference tree is present, the
    compiled reference) with oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", str(HERE), "ref"], check=True)


def _ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed to the oracle must be contiguous"
    return a.ctypes.data_as(_p)


class Config(C.Structure):
    """Layout of the reference's Config (common.h:187-265)."""
    _fields_ = [
        ("retain_device_mem", C.c_bool), ("num_major_cycles", _i), ("num_recievers", _i),
        ("num_baselines", _i), ("grid_size", _i), ("cell_size", _d), ("output_path", _p),
        ("dirty_image_output", _p), ("gpu_max_threads_per_block", _i),
        ("gpu_max_threads_per_block_dimension", _i), ("right_ascension", C.c_bool),
        ("save_dirty_image", C.c_bool), ("save_residual_image", C.c_bool),
        ("save_extracted_sources", C.c_bool), ("save_predicted_visibilities", C.c_bool),
        ("save_estimated_gains", C.c_bool), ("perform_system_test", C.c_bool),
        ("system_test_image", _p), ("system_test_sources", _p), ("system_test_visibilities", _p),
        ("system_test_gains", _p), ("default_gains_file", _p), ("output_gains_file", _p),
        ("perform_gain_calibration", C.c_bool), ("use_default_gains", C.c_bool),
        ("max_calibration_cycles", _i), ("number_cal_major_cycles", _i), ("force_weight_to_one", C.c_bool),
        ("frequency_hz", _d), ("oversampling", _i), ("uv_scale", _d), ("num_visibilities", _i),
        ("num_kernels", _i), ("total_kernel_samples", _i), ("max_w", _d), ("w_scale", _d),
        ("kernel_real_file", _p), ("kernel_imag_file", _p), ("kernel_support_file", _p),
        ("degridding_kernel_real_file", _p), ("degridding_kernel_imag_file", _p),
        ("degridding_kernel_support_file", _p), ("visibility_source_file", _p),
        ("number_minor_cycles_cal", C.c_uint), ("number_minor_cycles_img", C.c_uint), ("loop_gain", _d),
        ("weak_source_percent_gc", _d), ("weak_source_percent_img", _d), ("noise_factor", _d),
        ("psf_max_value", _d), ("model_sources_output", _p), ("residual_image_output", _p),
        ("psf_input_file", _p), ("psf_image_output", _p), ("clean_psf_image_output", _p),
        ("model_image_output", _p), ("final_image_output", _p), ("num_sources", _i),
        ("predicted_vis_output", _p),
    ]


assert C.sizeof(Config) == 360


def make_config(grid_size: int, uv_scale: float, w_scale: float, oversampling: int = 16,
                cell_size: float = 8.52211548825356e-06, psf_max_value: float = 0.0, loop_gain: float = 0.1,
                noise_factor: float = 1.5, weak_source_percent_img: float = 0.0002) -> Config:
    c = Config()
    c.grid_size = grid_size
    c.uv_scale = uv_scale
    c.w_scale = w_scale
    c.oversampling = oversampling
    c.cell_size = cell_size
    c.psf_max_value = psf_max_value
    c.loop_gain = loop_gain
    c.noise_factor = noise_factor
    c.weak_source_percent_img = weak_source_percent_img
    c.frequency_hz = 299792458.0
    c.right_ascension = True
    c.force_weight_to_one = True
    return c


class Oracle:
    """The C restatement.  precision: "f32" (reference default) or "f64"."""

    def __init__(self, precision: str = "f64"):
        self.precision = precision
        self.dtype = np.float32 if precision == "f32" else np.float64
        path = BUILD / f"liboracle_{precision}.so"
        if not path.exists():
            build()
        self.lib = C.CDLL(str(path))
        assert self.lib.or_real_size() == np.dtype(self.dtype).itemsize

    def _a(self, x, cols=None):
        a = np.ascontiguousarray(x, dtype=self.dtype)
        if cols is not None:
            a = a.reshape(-1, cols)
        return a

    def correct_to_finegrid(self, grid_size, os_, uvw, vis, uv_scale):
        uvw = self._a(uvw, 3)
        vis = self._a(vis, 2)
        n = uvw.shape[0]
        ov = np.empty_like(vis)
        ou = np.empty_like(uvw)
        cnt = _i(0)
        self.lib.or_correct_to_finegrid(_i(n), _i(grid_size), _i(os_), _ptr(uvw), _ptr(vis), _d(uv_scale),
                                        _ptr(ov), _ptr(ou), C.byref(cnt))
        return ov, ou, cnt.value

    def std_gridding(self, grid_size, os_, kernels, supports, uvw, vis, uv_scale, w_scale):
        k = self._a(kernels, 2)
        s = np.ascontiguousarray(supports, dtype=np.int32)
        uvw = self._a(uvw, 3)
        vis = self._a(vis, 2)
        grid = np.zeros((grid_size * grid_size, 2), dtype=self.dtype)
        self.lib.or_std_gridding(_i(grid_size), _i(os_), _i(uvw.shape[0]), _ptr(k), _ptr(s), _ptr(uvw), _ptr(vis),
                                 _d(uv_scale), _d(w_scale), _ptr(grid))
        return grid

    def std_degridding(self, grid_size, os_, kernels, supports, grid, uvw, uv_scale, w_scale, nearest=True):
        k = self._a(kernels, 2)
        s = np.ascontiguousarray(supports, dtype=np.int32)
        g = self._a(grid, 2)
        uvw = self._a(uvw, 3)
        out = np.zeros((uvw.shape[0], 2), dtype=self.dtype)
        self.lib.or_std_degridding(_i(grid_size), _i(os_), _i(uvw.shape[0]), _ptr(k), _ptr(s), _ptr(g), _ptr(uvw),
                                   _d(uv_scale), _d(w_scale), _ptr(out), _i(1 if nearest else 0))
        return out

    def g2g_degridgrid(self, grid_size, os_, gk, gs, dk, ds, in_grid, uvw, uv_scale):
        gk = self._a(gk, 2)
        dk = self._a(dk, 2)
        gs = np.ascontiguousarray(gs, dtype=np.int32)
        ds = np.ascontiguousarray(ds, dtype=np.int32)
        g = self._a(in_grid, 2)
        uvw = self._a(uvw, 3)
        out = np.zeros((grid_size * grid_size, 2), dtype=self.dtype)
        self.lib.or_g2g_degridgrid(_i(grid_size), _i(os_), _i(uvw.shape[0]), _ptr(gk), _ptr(gs), _ptr(dk), _ptr(ds),
                                   _ptr(g), _ptr(uvw), _d(uv_scale), _ptr(out))
        return out

    def gridding_cpu(self, grid_size, os_, kernels, supports, uvw, vis, uv_scale, w_scale, grid=None):
        k = self._a(kernels, 2)
        s = np.ascontiguousarray(supports, dtype=np.int32)
        uvw = self._a(uvw, 3)
        vis = self._a(vis, 2)
        if grid is None:
            grid = np.zeros((grid_size * grid_size, 2), dtype=self.dtype)
        else:
            grid = self._a(grid, 2).copy()
        self.lib.or_gridding_cpu(_ptr(grid), _ptr(k), _ptr(s), _ptr(uvw), _ptr(vis), _i(uvw.shape[0]), _i(os_),
                                 _i(grid_size), _d(uv_scale), _d(w_scale))
        return grid

    def subtract_vis(self, measured, predicted):
        m = self._a(measured, 2)
        p = self._a(predicted, 2)
        out = np.empty_like(m)
        self.lib.or_subtract_vis(_i(m.shape[0]), _ptr(m), _ptr(p), _ptr(out))
        return out

    def subtract_image(self, grid_size, a, b):
        a = self._a(a)
        b = self._a(b)
        out = np.empty_like(a)
        self.lib.or_subtract_image(_i(grid_size), _ptr(a), _ptr(b), _ptr(out))
        return out

    def fft_shift_c2c(self, grid_size, x):
        x = self._a(x, 2)
        out = np.empty_like(x)
        self.lib.or_fft_shift_c2c(_i(grid_size), _ptr(x), _ptr(out))
        return out

    def fft_shift_c2r(self, grid_size, x):
        x = self._a(x, 2)
        out = np.empty(x.shape[0], dtype=self.dtype)
        self.lib.or_fft_shift_c2r(_i(grid_size), _ptr(x), _ptr(out))
        return out

    def fft_shift_r2c(self, grid_size, x):
        x = self._a(x)
        out = np.empty((x.shape[0], 2), dtype=self.dtype)
        self.lib.or_fft_shift_r2c(_i(grid_size), _ptr(x), _ptr(out))
        return out

    def fft2d(self, grid_size, x, sign):
        x = self._a(x, 2)
        out = np.empty_like(x)
        self.lib.or_fft2d(_i(grid_size), _ptr(x), _ptr(out), _i(sign))
        return out

    def prolate_spheroidal(self, nu):
        self.lib.or_prolate_spheroidal.restype = _d
        return self.lib.or_prolate_spheroidal(_d(nu))

    def half_prolate(self, grid_size):
        """G/2 entries as the reference builds them, plus the (defined) entry G/2 = 0."""
        out = np.zeros(grid_size // 2 + 1, dtype=self.dtype)
        self.lib.or_create_1D_half_prolate(_ptr(out), _i(grid_size))
        return out

    def conv_correction(self, grid_size, image, prolate_ext):
        x = self._a(image)
        p = self._a(prolate_ext)
        assert p.shape[0] == grid_size // 2 + 1
        out = np.empty_like(x)
        self.lib.or_conv_correction(_i(grid_size), _ptr(x), _ptr(p), _ptr(out))
        return out

    def dft(self, sources, uvw):
        s = self._a(sources, 3)
        uvw = self._a(uvw, 3)
        out = np.empty((uvw.shape[0], 2), dtype=self.dtype)
        self.lib.or_dft(_i(uvw.shape[0]), _i(s.shape[0]), _ptr(s), _ptr(uvw), _ptr(out))
        return out

    def hogbom(self, grid_size, num_minor, max_sources, residual, psf, psf_max_value, cell_size, model=None,
               loop_gain=0.1, noise_factor=1.5, weak=0.0002):
        r = self._a(residual).reshape(-1)
        p = np.zeros(grid_size * grid_size + 1, dtype=self.dtype)
        p[:-1] = self._a(psf).reshape(-1)
        m = np.zeros_like(r) if model is None else self._a(model).reshape(-1)
        out_model = np.empty_like(r)
        out_res = np.empty_like(r)
        src = np.zeros((max(max_sources, num_minor), 3), dtype=self.dtype)
        n = _i(0)
        self.lib.or_hogbom_clean(_i(grid_size), _i(num_minor), _i(max_sources), _ptr(r), _ptr(p), _d(loop_gain),
                                 _d(noise_factor), _d(weak), _d(psf_max_value), _d(cell_size), _ptr(m), C.byref(n),
                                 _ptr(src), _ptr(out_model), _ptr(out_res))
        return n.value, src[:n.value].copy(), out_model, out_res

    def merge_grids(self, grid_size, grids):
        g = self._a(grids, 2)
        slices = g.shape[0] // (grid_size * grid_size)
        out = np.empty((grid_size * grid_size, 2), dtype=self.dtype)
        self.lib.or_merge_grids(_i(grid_size), _i(slices), _ptr(g), _ptr(out))
        return out

    def psf_crop_normalise(self, grid_size, full_psf):
        f = self._a(full_psf).reshape(-1)
        pg = int(round(np.sqrt(f.shape[0])))
        out = np.empty(grid_size * grid_size, dtype=self.dtype)
        self.lib.or_psf_crop_normalise.restype = _d
        mx = self.lib.or_psf_crop_normalise(_i(grid_size), _i(pg), _ptr(f), _ptr(out))
        return mx, out

    def clean_psf(self, grid_size, psf_max_value, dirty_psf):
        d = self._a(dirty_psf).reshape(-1)
        out = np.empty_like(d)
        hd = np.zeros(2, dtype=np.int32)
        self.lib.or_clean_psf(_i(grid_size), _d(psf_max_value), _ptr(d), _ptr(out), _ptr(hd))
        return out, hd


class RefLib:
    """The reference's actor sources compiled unmodified (oracle/_ref).

    ``variant`` "parity" is the -O2, no-FMA build used to pin the oracle;
    "fast" is the -O3 AVX2/FMA float build used only for timing."""

    def __init__(self, precision: str = "f32", variant: str = "parity"):
        self.precision = precision
        self.dtype = np.float32 if precision == "f32" else np.float64
        name = f"libref_{precision}.so" if variant == "parity" else f"libref_{precision}_fast.so"
        path = REFDIR / name
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle ref, needs the reference tree)")
        self.lib = C.CDLL(str(path))
        self.lib.prolate_spheroidal.restype = _d

    @staticmethod
    def available(precision: str = "f32", variant: str = "parity") -> bool:
        name = f"libref_{precision}.so" if variant == "parity" else f"libref_{precision}_fast.so"
        return (REFDIR / name).exists()

    def _a(self, x, cols=None):
        a = np.ascontiguousarray(x, dtype=self.dtype)
        if cols is not None:
            a = a.reshape(-1, cols)
        return a

    def std_gridding(self, cfg: Config, grid_size, os_, kernels, supports, uvw, vis, num=None, out=None):
        """out: an optional preallocated (G^2, 2) grid of this precision (the
        reference clears it itself, degridgrid.c:73)."""
        k = self._a(kernels, 2)
        s = np.ascontiguousarray(supports, dtype=np.int32)
        uvw = self._a(uvw, 3)
        vis = self._a(vis, 2)
        n = uvw.shape[0] if num is None else num
        nk = s.shape[0]
        if out is not None:
            assert out.dtype == self.dtype and out.shape == (grid_size * grid_size, 2) and out.flags["C_CONTIGUOUS"]
            grid = out
        else:
            grid = np.zeros((grid_size * grid_size, 2), dtype=self.dtype)
        maj = _i(0)
        nc = _i(n)
        self.lib.std_gridding(_i(grid_size), _i(n), _i(nk), _i(k.shape[0]), _i(os_), _i(0), C.byref(maj),
                              C.byref(nc), _ptr(k), _ptr(s), _ptr(uvw), _ptr(vis), C.byref(cfg), None, _ptr(grid))
        return grid

    def padded_grid(self, grid_size, grid):
        """The grid with 2 G zero rows appended: the nearest-cell read
        (degridgrid.c:194-199) has no bounds check, and a point at the top edge
        reads past the grid; the zero rows make that read defined (0), the value
        the oracle assigns."""
        g = np.zeros((grid_size * grid_size + 2 * grid_size, 2), dtype=self.dtype)
        g[: grid_size * grid_size] = self._a(grid, 2)
        return g

    def std_degridding(self, cfg: Config, grid_size, os_, kernels, supports, grid, uvw, num=None, padded=False):
        """padded: grid already comes from padded_grid (no per-call copy)."""
        k = self._a(kernels, 2)
        s = np.ascontiguousarray(supports, dtype=np.int32)
        if padded:
            assert grid.dtype == self.dtype and grid.shape == (grid_size * grid_size + 2 * grid_size, 2)
            g = grid
        else:
            g = self.padded_grid(grid_size, grid)
        uvw = self._a(uvw, 3)
        n = uvw.shape[0] if num is None else num
        out = np.zeros((uvw.shape[0], 2), dtype=self.dtype)
        nc = _i(n)
        self.lib.std_degridding(_i(grid_size), _i(n), _i(s.shape[0]), _i(k.shape[0]), _i(os_), _ptr(k), _ptr(s),
                                _ptr(g), _ptr(uvw), C.byref(nc), C.byref(cfg), _ptr(out))
        return out

    def subtract_finegrid(self, measured, predicted, num=None):
        m = self._a(measured, 2)
        p = self._a(predicted, 2)
        n = m.shape[0] if num is None else num
        out = np.zeros_like(m)
        nc = _i(n)
        self.lib.subtract_from_measurements_finegrid(_i(n), _ptr(m), _ptr(p), C.byref(nc), _ptr(out))
        return out

    def g2g_degridgrid(self, cfg: Config, grid_size, os_, gk, gs, dk, ds, in_grid, uvw):
        gk = self._a(gk, 2)
        dk = self._a(dk, 2)
        gs = np.ascontiguousarray(gs, dtype=np.int32)
        ds = np.ascontiguousarray(ds, dtype=np.int32)
        # as in std_degridding: the nearest-cell read (degridgrid.c:273-279) is
        # only checked below; zero rows past the grid make it defined
        g = np.zeros((grid_size * grid_size + 2 * grid_size, 2), dtype=self.dtype)
        g[: grid_size * grid_size] = self._a(in_grid, 2)
        uvw = self._a(uvw, 3)
        out = np.zeros((grid_size * grid_size, 2), dtype=self.dtype)
        nc = _i(uvw.shape[0])
        self.lib.g2g_degridgrid(_i(grid_size), _i(uvw.shape[0]), _i(gs.shape[0]), _i(ds.shape[0]), _i(gk.shape[0]),
                                _i(dk.shape[0]), _i(os_), _ptr(gk), _ptr(gs), _ptr(dk), _ptr(ds), _ptr(g), _ptr(uvw),
                                C.byref(nc), C.byref(cfg), _ptr(out))
        return out

    def gridding_actor(self, cfg: Config, grid_size, kernels, supports, uvw, vis):
        k = self._a(kernels, 2)
        s = np.ascontiguousarray(supports, dtype=np.int32)
        uvw = self._a(uvw, 3)
        vis = self._a(vis, 2)
        grid = np.zeros((grid_size * grid_size, 2), dtype=self.dtype)
        self.lib.gridding_actor(_i(grid_size), _i(uvw.shape[0]), _i(s.shape[0]), _i(k.shape[0]), _ptr(k), _ptr(s),
                                _ptr(uvw), _ptr(vis), C.byref(cfg), _ptr(grid))
        return grid

    def correct_to_finegrid(self, cfg: Config, grid_size, os_, uvw, vis):
        uvw = self._a(uvw, 3)
        vis = self._a(vis, 2)
        n = uvw.shape[0]
        ov = np.zeros_like(vis)
        ou = np.zeros_like(uvw)
        cnt = _i(0)
        self.lib.correct_to_finegrid(_i(n), _i(grid_size), _i(os_), _i(0), _ptr(uvw), _ptr(vis), C.byref(cfg),
                                     _ptr(ov), _ptr(ou), C.byref(cnt))
        return ov, ou, cnt.value

    def fft_shift_c2c(self, cfg, grid_size, x):
        x = self._a(x, 2)
        out = np.empty_like(x)
        self.lib.fft_shift_complex_to_complex_actor(_i(grid_size), _ptr(x), C.byref(cfg), _ptr(out))
        return out

    def fft_shift_c2r(self, cfg, grid_size, x):
        x = self._a(x, 2)
        out = np.empty(x.shape[0], dtype=self.dtype)
        self.lib.fft_shift_complex_to_real_actor(_i(grid_size), _ptr(x), C.byref(cfg), _ptr(out))
        return out

    def fft_shift_r2c(self, cfg, grid_size, x):
        x = self._a(x)
        out = np.empty((x.shape[0], 2), dtype=self.dtype)
        self.lib.fft_shift_real_to_complex_actor(_i(grid_size), _ptr(x), C.byref(cfg), _ptr(out))
        return out

    def fft(self, grid_size, x, inverse):
        x = self._a(x, 2)
        out = np.empty_like(x)
        fn = self.lib.CUFFT_EXECUTE_INVERSE_C2C_actor if inverse else self.lib.CUFFT_EXECUTE_FORWARD_C2C_actor
        fn(_i(grid_size), _ptr(x), _ptr(out))
        return out

    def half_prolate_ext(self, grid_size):
        out = np.zeros(grid_size // 2 + 1, dtype=self.dtype)
        self.lib.create_1D_half_prolate(_ptr(out), _i(grid_size))
        return out

    def conv_correction(self, cfg, grid_size, image, prolate_ext):
        x = self._a(image)
        p = self._a(prolate_ext)
        out = np.empty_like(x)
        self.lib.execute_convolution_correction_actor(_i(grid_size), _ptr(x), _ptr(p), C.byref(cfg), _ptr(out))
        return out

    def dft(self, cfg, sources, uvw):
        s = self._a(sources, 3)
        uvw = self._a(uvw, 3)
        out = np.empty((uvw.shape[0], 2), dtype=self.dtype)
        ns = _i(s.shape[0])
        self.lib.dft_actor(_i(uvw.shape[0]), _i(s.shape[0]), _ptr(s), _ptr(uvw), C.byref(ns), C.byref(cfg),
                           _ptr(out))
        return out

    def hogbom(self, cfg, grid_size, num_minor, max_sources, residual, psf, model=None):
        r = self._a(residual).reshape(-1).copy()
        p = np.zeros(grid_size * grid_size + 1, dtype=self.dtype)   # one defined entry past the end
        p[:-1] = self._a(psf).reshape(-1)
        m = np.zeros_like(r) if model is None else self._a(model).reshape(-1).copy()
        out_model = np.empty_like(r)
        src = np.zeros((max(max_sources, num_minor), 3), dtype=self.dtype)
        n = _i(0)
        hd = np.zeros(2, dtype=np.int32)
        self.lib.hogbom_clean(_i(grid_size), _i(num_minor), _i(max_sources), _ptr(r), _ptr(p), _ptr(hd),
                              C.byref(cfg), _ptr(m), C.byref(n), _ptr(src), _ptr(out_model))
        return n.value, src[:n.value].copy(), out_model

    def merge_grids(self, grid_size, grids):
        g = self._a(grids, 2)
        slices = g.shape[0] // (grid_size * grid_size)
        out = np.empty((grid_size * grid_size, 2), dtype=self.dtype)
        self.lib.merge_gridded_visibilities(_i(grid_size), _i(slices), _ptr(g), _ptr(out))
        return out

    def subtract_image(self, grid_size, a, b):
        a = self._a(a)
        b = self._a(b)
        out = np.empty_like(a)
        self.lib.subtract_image_space(_i(grid_size), _ptr(a), _ptr(b), _ptr(out))
        return out

    def clean_psf(self, cfg, grid_size, dirty_psf):
        d = self._a(dirty_psf).reshape(-1)
        out = np.empty_like(d)
        hd = np.zeros(2, dtype=np.int32)
        self.lib.clean_psf_host_set_up(_i(grid_size), _i(1), C.byref(cfg), _ptr(d), _ptr(out), _ptr(hd))
        return out, hd


def fft_pipeline(o: Oracle, G, OS, uvw_raw, vis, gk, dk, supports, uv_scale, w_scale, psf, psf_max, cell,
                 cycles, minor, max_sources, nearest=True, loop_gain=0.1, noise_factor=1.5, weak=0.0002):
    """The FFT pipeline's major cycles in the order of the generated schedule
    (code_fft_1core/generated/Core0.c: correct_to_finegrid :3101 once, then
    per cycle the model -> inverse taper (identity) -> fft_shift r2c -> FFTW
    forward -> fft_shift c2c -> std_degridding -> subtract -> std_gridding ->
    fft_shift c2c -> FFTW backward -> fft_shift c2r -> taper -> hogbom_clean),
    with the live Hogbom and one visibility slice (the schedule's four slices
    only split the same sums).  Returns per cycle (residual image, model
    image, number of components, components)."""
    _, uvw_c, _ = o.correct_to_finegrid(G, OS, uvw_raw, vis, uv_scale)
    prolate = o.half_prolate(G)
    model = np.zeros(G * G, dtype=o.dtype)
    out = []
    for _ in range(cycles):
        mg = o.fft_shift_c2c(G, o.fft2d(G, o.fft_shift_r2c(G, model), -1))
        pred = o.std_degridding(G, OS, dk, supports, mg, uvw_c, uv_scale, w_scale, nearest=nearest)
        delta = o.subtract_vis(vis, pred)
        rg = o.std_gridding(G, OS, gk, supports, uvw_c, delta, uv_scale, w_scale)
        img = o.conv_correction(G, o.fft_shift_c2r(G, o.fft2d(G, o.fft_shift_c2c(G, rg), +1)), prolate)
        n, src, model, _ = o.hogbom(G, minor, max_sources, img, psf, psf_max, cell, model=model,
                                    loop_gain=loop_gain, noise_factor=noise_factor, weak=weak)
        out.append((img.copy(), model.copy(), n, src))
    return out


def dirty_psf(o: Oracle, G, OS, uvw_raw, gk, supports, uv_scale, w_scale):
    """PSF of the array as the pipeline images it: unit visibilities gridded,
    transformed and taper-corrected, then cropped and normalised as
    psf_host_set_up does (top.c:453-515).  Returns (psf, psf_max)."""
    ones = np.zeros((uvw_raw.shape[0], 2), dtype=o.dtype)
    ones[:, 0] = 1.0
    _, uvw_c, _ = o.correct_to_finegrid(G, OS, uvw_raw, ones, uv_scale)
    g = o.std_gridding(G, OS, gk, supports, uvw_c, ones, uv_scale, w_scale)
    img = o.conv_correction(G, o.fft_shift_c2r(G, o.fft2d(G, o.fft_shift_c2c(G, g), +1)), o.half_prolate(G))
    mx, psf = o.psf_crop_normalise(G, img)
    return psf, mx
