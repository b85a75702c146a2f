"""ctypes front end of libsdp_b200.so.

Two layers, matching include/sdp_b200.h:

* ``Actors``: the reference's PREESM actors (host numpy arrays in, host
  numpy arrays out), called through the exported C symbols exactly as the
  generated schedule calls them.  Method names and argument order follow the
  reference actors (param_code/code_*_1core/include/*.h).
* ``Device``: the device-resident sdp_* layer on torch CUDA tensors (torch is
  used only to own device memory and streams; every computation is a kernel
  of libsdp_b200.so).

Loading fails loudly when the library is missing; there is no fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libsdp_b200.so"
HEADER = HERE.parent / "include" / "sdp_b200.h"

SDP_OK = 0
SDP_ERR_INVALID = 1
SDP_ERR_RANGE = 2
SDP_ERR_CUDA = 3
SDP_ERR_NOMEM = 4
SDP_ERR_TIMEOUT = 5
SDP_ERR_DATA = 6
SDP_ERR_IO = 7
SDP_DEGRID_NEAREST = 0
SDP_DEGRID_CONV = 1
SDP_GRID_STD = 0
SDP_GRID_SNAPPED = 1
SDP_GRID_G2G = 2

_i = C.c_int
_d = C.c_double
_p = C.c_void_p
_sz = C.c_size_t


class SdpError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"sdp status {status}: {message}")
        self.status = status


class Config(C.Structure):
    """Layout of the reference's Config (common.h:187-265) == sdp_config."""
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


class Geometry(C.Structure):
    _fields_ = [("grid_size", _i), ("oversampling", _i), ("uv_scale", _d), ("w_scale", _d)]


class WKernels(C.Structure):
    _fields_ = [("kernels", _p), ("supports", _p), ("num_kernels", _i), ("total_samples", _i),
                ("max_half_support", _i)]


class CleanParams(C.Structure):
    _fields_ = [("grid_size", _i), ("num_minor_cycles", _i), ("max_sources", _i), ("loop_gain", _d),
                ("noise_factor", _d), ("weak_source_percent", _d), ("psf_max_value", _d), ("cell_size", _d)]


def header_functions(header: Path = HEADER) -> list[str]:
    """Names of every function declared in include/sdp_b200.h."""
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s*([A-Za-z_][A-Za-z0-9_]*)\s*\(",
                       text, flags=re.M)
    return [n for n in names if n not in ("if", "for", "while", "return", "sizeof")]


_lib = None


def load(path: Path | str | None = None) -> C.CDLL:
    """Loads libsdp_b200.so (raises when it is missing: there is no fallback)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is not built; run python {HERE / 'build.py'}")
    lib = C.CDLL(str(p))
    lib.sdp_last_error.restype = C.c_char_p
    lib.prolate_spheroidal.restype = _d
    lib.prolate_spheroidal.argtypes = [_d]
    for name in ("sdp_visplan_create",):
        getattr(lib, name).restype = _i
    lib.gridding_CPU.argtypes = [_p, _p, _p, _p, _p, _i, _i, _i, _d, _d]
    if path is None:
        _lib = lib
    return lib


def check(status: int, lib: C.CDLL | None = None) -> None:
    if status != SDP_OK:
        lib = lib or load()
        raise SdpError(status, lib.sdp_last_error().decode())


def _ptr(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_p)


def _f32(x, cols=None):
    a = np.ascontiguousarray(x, dtype=np.float32)
    if cols is not None:
        a = a.reshape(-1, cols)
    return a


# ---------------------------------------------------------------------------
# Binary input files (sdp_bin_*)
# ---------------------------------------------------------------------------
_ll = C.c_longlong


def bin_info(path, lib: C.CDLL | None = None):
    """(kind, count, aux) of an sdp binary file."""
    lib = lib or load()
    k, n, a = _i(0), _ll(0), _ll(0)
    check(lib.sdp_bin_info(str(path).encode(), C.byref(k), C.byref(n), C.byref(a)), lib)
    return k.value, n.value, a.value


def bin_write_vis(path, uvw, vis, snapped=False, lib: C.CDLL | None = None):
    lib = lib or load()
    u, v = _f32(uvw, 3), _f32(vis, 2)
    assert u.shape[0] == v.shape[0]
    check(lib.sdp_bin_write_vis(str(path).encode(), _ll(u.shape[0]), _ptr(u), _ptr(v), _i(1 if snapped else 0)), lib)


def bin_write_kernels(path, supports, samples, lib: C.CDLL | None = None):
    lib = lib or load()
    s = np.ascontiguousarray(supports, dtype=np.int32).reshape(-1, 2)
    k = _f32(samples, 2)
    check(lib.sdp_bin_write_kernels(str(path).encode(), _i(s.shape[0]), _ll(k.shape[0]), _ptr(s), _ptr(k)), lib)


def bin_write_image(path, image, lib: C.CDLL | None = None):
    lib = lib or load()
    a = _f32(image)
    assert a.ndim == 2
    check(lib.sdp_bin_write_image(str(path).encode(), _i(a.shape[0]), _i(a.shape[1]), _ptr(a)), lib)


def bin_read_vis_host(path, lib: C.CDLL | None = None):
    """(uvw, vis, snapped) read into host arrays."""
    lib = lib or load()
    _, n, _ = bin_info(path, lib)
    u = np.empty((n, 3), np.float32)
    v = np.empty((n, 2), np.float32)
    got, sn = _ll(0), _i(0)
    check(lib.sdp_bin_read_vis_host(str(path).encode(), _ll(n), _ptr(u), _ptr(v), C.byref(got), C.byref(sn)), lib)
    return u, v, bool(sn.value)


# ---------------------------------------------------------------------------
# Actor layer (host arrays)
# ---------------------------------------------------------------------------
class Actors:
    """Calls the exported actor symbols the way the PREESM schedule does."""

    def __init__(self, lib: C.CDLL | None = None):
        self.lib = lib or load()

    def _status(self):
        st = self.lib.sdp_last_status()
        if st != SDP_OK:
            msg = self.lib.sdp_last_error().decode()
            self.lib.sdp_clear_error()
            raise SdpError(st, msg)

    def set_degrid_mode(self, mode: int):
        check(self.lib.sdp_set_degrid_mode(_i(mode)), self.lib)

    def std_gridding(self, cfg: Config, grid_size, os_, kernels, supports, uvw, vis, num=None, out=None):
        k = _f32(kernels, 2)
        s = np.ascontiguousarray(supports, dtype=np.int32)
        uvw = _f32(uvw, 3)
        vis = _f32(vis, 2)
        n = uvw.shape[0] if num is None else num
        grid = np.empty((grid_size * grid_size, 2), dtype=np.float32) if out is None else out
        maj = _i(0)
        nc = _i(n)
        self.lib.sdp_clear_error()
        self.lib.std_gridding(_i(grid_size), _i(uvw.shape[0]), _i(s.shape[0]), _i(k.shape[0]), _i(os_), _i(0),
                              C.byref(maj), C.byref(nc), _ptr(k), _ptr(s), _ptr(uvw), _ptr(vis), C.byref(cfg), None,
                              _ptr(grid))
        self._status()
        return grid

    def std_degridding(self, cfg: Config, grid_size, os_, kernels, supports, grid, uvw, num=None, out=None):
        k = _f32(kernels, 2)
        s = np.ascontiguousarray(supports, dtype=np.int32)
        g = _f32(grid, 2)
        uvw = _f32(uvw, 3)
        n = uvw.shape[0] if num is None else num
        o = np.empty((uvw.shape[0], 2), dtype=np.float32) if out is None else out
        nc = _i(n)
        self.lib.sdp_clear_error()
        self.lib.std_degridding(_i(grid_size), _i(uvw.shape[0]), _i(s.shape[0]), _i(k.shape[0]), _i(os_), _ptr(k),
                                _ptr(s), _ptr(g), _ptr(uvw), C.byref(nc), C.byref(cfg), _ptr(o))
        self._status()
        return o

    def subtract_finegrid(self, measured, predicted, num=None, out=None):
        m = _f32(measured, 2)
        p = _f32(predicted, 2)
        n = m.shape[0] if num is None else num
        o = np.zeros_like(m) if out is None else out
        nc = _i(n)
        self.lib.sdp_clear_error()
        self.lib.subtract_from_measurements_finegrid(_i(m.shape[0]), _ptr(m), _ptr(p), C.byref(nc), _ptr(o))
        self._status()
        return o

    def g2g_degridgrid(self, cfg: Config, grid_size, os_, gk, gs, dk, ds, in_grid, uvw):
        gk = _f32(gk, 2)
        dk = _f32(dk, 2)
        gs = np.ascontiguousarray(gs, dtype=np.int32)
        ds = np.ascontiguousarray(ds, dtype=np.int32)
        g = _f32(in_grid, 2)
        uvw = _f32(uvw, 3)
        out = np.empty((grid_size * grid_size, 2), dtype=np.float32)
        nc = _i(uvw.shape[0])
        self.lib.sdp_clear_error()
        self.lib.g2g_degridgrid(_i(grid_size), _i(uvw.shape[0]), _i(gs.shape[0]), _i(ds.shape[0]), _i(gk.shape[0]),
                                _i(dk.shape[0]), _i(os_), _ptr(gk), _ptr(gs), _ptr(dk), _ptr(ds), _ptr(g), _ptr(uvw),
                                C.byref(nc), C.byref(cfg), _ptr(out))
        self._status()
        return out

    def gridding_actor(self, cfg: Config, grid_size, kernels, supports, uvw, vis):
        k = _f32(kernels, 2)
        s = np.ascontiguousarray(supports, dtype=np.int32)
        uvw = _f32(uvw, 3)
        vis = _f32(vis, 2)
        grid = np.empty((grid_size * grid_size, 2), dtype=np.float32)
        self.lib.sdp_clear_error()
        self.lib.gridding_actor(_i(grid_size), _i(uvw.shape[0]), _i(s.shape[0]), _i(k.shape[0]), _ptr(k), _ptr(s),
                                _ptr(uvw), _ptr(vis), C.byref(cfg), _ptr(grid))
        self._status()
        return grid

    def gridding_cpu(self, grid, kernels, supports, uvw, vis, os_, grid_size, uv_scale, w_scale):
        g = _f32(grid, 2).copy()
        k = _f32(kernels, 2)
        s = np.ascontiguousarray(supports, dtype=np.int32)
        uvw = _f32(uvw, 3)
        vis = _f32(vis, 2)
        self.lib.sdp_clear_error()
        self.lib.gridding_CPU(_ptr(g), _ptr(k), _ptr(s), _ptr(uvw), _ptr(vis), uvw.shape[0], os_, grid_size,
                              uv_scale, w_scale)
        self._status()
        return g

    def correct_to_finegrid(self, cfg: Config, grid_size, os_, uvw, vis, simplify=0):
        uvw = _f32(uvw, 3)
        vis = _f32(vis, 2)
        n = uvw.shape[0]
        ov = np.zeros_like(vis)
        ou = np.zeros_like(uvw)
        cnt = _i(0)
        self.lib.sdp_clear_error()
        self.lib.correct_to_finegrid(_i(n), _i(grid_size), _i(os_), _i(simplify), _ptr(uvw), _ptr(vis),
                                     C.byref(cfg), _ptr(ov), _ptr(ou), C.byref(cnt))
        self._status()
        return ov, ou, cnt.value

    def fft_shift_c2c(self, cfg, grid_size, x):
        x = _f32(x, 2)
        out = np.empty_like(x)
        self.lib.sdp_clear_error()
        self.lib.fft_shift_complex_to_complex_actor(_i(grid_size), _ptr(x), C.byref(cfg), _ptr(out))
        self._status()
        return out

    def fft_shift_c2r(self, cfg, grid_size, x):
        x = _f32(x, 2)
        out = np.empty(x.shape[0], dtype=np.float32)
        self.lib.sdp_clear_error()
        self.lib.fft_shift_complex_to_real_actor(_i(grid_size), _ptr(x), C.byref(cfg), _ptr(out))
        self._status()
        return out

    def fft_shift_r2c(self, cfg, grid_size, x):
        x = _f32(x)
        out = np.empty((x.shape[0], 2), dtype=np.float32)
        self.lib.sdp_clear_error()
        self.lib.fft_shift_real_to_complex_actor(_i(grid_size), _ptr(x), C.byref(cfg), _ptr(out))
        self._status()
        return out

    def fft(self, grid_size, x, inverse):
        x = _f32(x, 2)
        out = np.empty_like(x)
        fn = self.lib.CUFFT_EXECUTE_INVERSE_C2C_actor if inverse else self.lib.CUFFT_EXECUTE_FORWARD_C2C_actor
        self.lib.sdp_clear_error()
        fn(_i(grid_size), _ptr(x), _ptr(out))
        self._status()
        return out

    def half_prolate(self, grid_size):
        out = np.zeros(grid_size // 2, dtype=np.float32)
        self.lib.sdp_clear_error()
        self.lib.create_1D_half_prolate(_ptr(out), _i(grid_size))
        self._status()
        return out

    def conv_correction(self, cfg, grid_size, image, prolate):
        x = _f32(image)
        p = _f32(prolate)[: grid_size // 2].copy()
        out = np.empty_like(x)
        self.lib.sdp_clear_error()
        self.lib.execute_convolution_correction_actor(_i(grid_size), _ptr(x), _ptr(p), C.byref(cfg), _ptr(out))
        self._status()
        return out

    def dft(self, cfg, sources, uvw):
        s = _f32(sources, 3)
        uvw = _f32(uvw, 3)
        out = np.empty((uvw.shape[0], 2), dtype=np.float32)
        ns = _i(s.shape[0])
        self.lib.sdp_clear_error()
        self.lib.dft_actor(_i(uvw.shape[0]), _i(s.shape[0]), _ptr(s), _ptr(uvw), C.byref(ns), C.byref(cfg), _ptr(out))
        self._status()
        return out

    def hogbom(self, cfg, grid_size, num_minor, max_sources, residual, psf, model=None):
        r = _f32(residual).reshape(-1)
        p = _f32(psf).reshape(-1)
        m = np.zeros_like(r) if model is None else _f32(model).reshape(-1)
        out_model = np.empty_like(r)
        src = np.zeros((max(max_sources, 1), 3), dtype=np.float32)
        n = _i(0)
        hd = np.zeros(2, dtype=np.int32)
        self.lib.sdp_clear_error()
        self.lib.hogbom_clean(_i(grid_size), _i(num_minor), _i(max_sources), _ptr(r), _ptr(p), _ptr(hd), C.byref(cfg),
                              _ptr(m), C.byref(n), _ptr(src), _ptr(out_model))
        self._status()
        return n.value, src[:n.value].copy(), out_model

    def merge_grids(self, grid_size, grids):
        g = _f32(grids, 2)
        slices = g.shape[0] // (grid_size * grid_size)
        out = np.empty((grid_size * grid_size, 2), dtype=np.float32)
        self.lib.sdp_clear_error()
        self.lib.merge_gridded_visibilities(_i(grid_size), _i(slices), _ptr(g), _ptr(out))
        self._status()
        return out

    def subtract_image(self, grid_size, a, b):
        a = _f32(a)
        b = _f32(b)
        out = np.empty_like(a)
        self.lib.sdp_clear_error()
        self.lib.subtract_image_space(_i(grid_size), _ptr(a), _ptr(b), _ptr(out))
        self._status()
        return out

    def add_visibilities(self, a, b):
        a = _f32(a, 2)
        b = _f32(b, 2)
        out = np.empty_like(a)
        self.lib.sdp_clear_error()
        self.lib.add_visibilities(_i(a.shape[0]), _ptr(a), _ptr(b), _ptr(out))
        self._status()
        return out

    def clean_psf(self, cfg, grid_size, dirty_psf):
        d = _f32(dirty_psf).reshape(-1)
        out = np.empty_like(d)
        hd = np.zeros(2, dtype=np.int32)
        self.lib.sdp_clear_error()
        self.lib.clean_psf_host_set_up(_i(grid_size), _i(1), C.byref(cfg), _ptr(d), _ptr(out), _ptr(hd))
        self._status()
        return out, hd


# ---------------------------------------------------------------------------
# Device layer (torch CUDA tensors)
# ---------------------------------------------------------------------------
def _dp(t):
    """Device pointer of a contiguous torch tensor (or None)."""
    if t is None:
        return None
    assert t.is_cuda and t.is_contiguous()
    return _p(t.data_ptr())


def _stream(s=None):
    import torch
    s = s if s is not None else torch.cuda.current_stream()
    return _p(s.cuda_stream)


class PlanOptions(C.Structure):
    """Plan shape: uv tile side, visibilities per work item, lanes per
    visibility (0: the warp-per-visibility kernel where it applies), warps per
    CTA of that kernel (0 = by occupancy)."""
    _fields_ = [("tile", _i), ("chunk", _i), ("lanes", _i), ("warps", _i)]


class VisPlan:
    """Owns an sdp_visplan (visibilities binned by uv tile and w-plane)."""

    def __init__(self, lib, geom: Geometry, gk: WKernels, dk: WKernels | None, uvw, mode: int, stream=None,
                 keep=(), options: PlanOptions | None = None):
        self.lib = lib
        self.geom = geom
        self._keep = keep  # tensors the plan points at
        self.gk = gk
        self.dk = dk or gk
        self.n = int(uvw.shape[0])
        self.handle = _p()
        if options is None:
            check(lib.sdp_visplan_create(C.byref(self.handle), C.byref(geom), C.byref(self.gk), C.byref(self.dk),
                                         _i(self.n), _dp(uvw), _i(mode), _stream(stream)), lib)
        else:
            check(lib.sdp_visplan_create_opt(C.byref(self.handle), C.byref(geom), C.byref(self.gk),
                                             C.byref(self.dk), _i(self.n), _dp(uvw), _i(mode), C.byref(options),
                                             _stream(stream)), lib)

    def options(self) -> PlanOptions:
        o = PlanOptions()
        check(self.lib.sdp_visplan_options(self.handle, C.byref(o)), self.lib)
        return o

    def close(self):
        if self.handle:
            check(self.lib.sdp_visplan_destroy(self.handle), self.lib)
            self.handle = _p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def num_work_items(self) -> int:
        c = _i(0)
        check(self.lib.sdp_visplan_num_work_items(self.handle, C.byref(c)), self.lib)
        return c.value

    def set_measured(self, vis, stream=None):
        check(self.lib.sdp_visplan_set_measured(self.handle, _dp(vis), _stream(stream)), self.lib)

    def grid(self, vis, grid, accumulate=False, stream=None):
        check(self.lib.sdp_visplan_grid(self.handle, _dp(vis), _dp(grid), _i(1 if accumulate else 0),
                                        _stream(stream)), self.lib)

    def degrid(self, model_grid, predicted, mode=SDP_DEGRID_CONV, stream=None):
        check(self.lib.sdp_visplan_degrid(self.handle, _dp(model_grid), _dp(predicted), _i(mode), _stream(stream)),
              self.lib)

    def cycle(self, model_grid, residual_grid, mode=SDP_DEGRID_CONV, predicted=None, delta=None, stream=None):
        check(self.lib.sdp_visplan_cycle(self.handle, _dp(model_grid), _i(mode), _dp(predicted), _dp(delta),
                                         _dp(residual_grid), _stream(stream)), self.lib)

    def g2g(self, in_grid, out_grid, stream=None):
        check(self.lib.sdp_visplan_g2g(self.handle, _dp(in_grid), _dp(out_grid), _stream(stream)), self.lib)

    def check_flags(self, stream=None):
        check(self.lib.sdp_visplan_check(self.handle, _stream(stream)), self.lib)


class VisBatch:
    """Owns an sdp_visbatch: several channels' plans in one launch.  The plans
    (VisPlan objects) are kept alive by the batch."""

    def __init__(self, lib, plans, stream=None):
        self.lib = lib
        self.plans = list(plans)
        arr = (_p * len(self.plans))(*[pl.handle for pl in self.plans])
        self.handle = _p()
        check(lib.sdp_visbatch_create(C.byref(self.handle), arr, _i(len(self.plans)), _stream(stream)), lib)
        self._grids = ()

    def set_grids(self, model_grids, residual_grids, stream=None):
        n = len(self.plans)
        m = (_p * n)(*[_dp(g) for g in model_grids])
        r = (_p * n)(*[_dp(g) for g in residual_grids])
        self._grids = (list(model_grids), list(residual_grids))
        check(self.lib.sdp_visbatch_set_grids(self.handle, m, r, _stream(stream)), self.lib)

    def cycle(self, mode=SDP_DEGRID_CONV, stream=None):
        check(self.lib.sdp_visbatch_cycle(self.handle, _i(mode), _stream(stream)), self.lib)

    def num_work_items(self) -> int:
        c = _i(0)
        check(self.lib.sdp_visbatch_num_work_items(self.handle, C.byref(c)), self.lib)
        return c.value

    def close(self):
        if self.handle:
            check(self.lib.sdp_visbatch_destroy(self.handle), self.lib)
            self.handle = _p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


SDP_COORD_F32 = 0
SDP_COORD_F64 = 1
SDP_PLAN_COORD_F64 = 0x100
SDP_PLAN_SNAP = 0x200


class PipelineConfig(C.Structure):
    _fields_ = [("grid_size", _i), ("oversampling", _i), ("uv_scale", _d), ("w_scale", _d), ("cell_size", _d),
                ("num_minor_cycles", _i), ("max_sources", _i), ("loop_gain", _d), ("noise_factor", _d),
                ("weak_source_percent", _d), ("psf_max_value", _d), ("degrid_mode", _i), ("coord_mode", _i),
                ("snap", _i), ("use_graph", _i)]


class Pipeline:
    """Owns an sdp_pipeline: the device-resident FFT-pipeline major cycle."""

    def __init__(self, lib, cfg: PipelineConfig, gk: WKernels, dk: WKernels | None, uvw, measured, psf,
                 stream=None, keep=()):
        self.lib = lib
        self.cfg = cfg
        self._keep = keep
        self.handle = _p()
        self.G = cfg.grid_size
        check(lib.sdp_pipeline_create(C.byref(self.handle), C.byref(cfg), C.byref(gk),
                                      C.byref(dk) if dk is not None else None, _i(int(uvw.shape[0])), _dp(uvw),
                                      _dp(measured), _dp(psf), _stream(stream)), lib)

    def major_cycle(self, stream=None):
        check(self.lib.sdp_pipeline_major_cycle(self.handle, _stream(stream)), self.lib)

    def graph_active(self) -> bool:
        return bool(self.lib.sdp_pipeline_graph_active(self.handle))

    def graph_error(self) -> str:
        self.lib.sdp_pipeline_graph_error.restype = C.c_char_p
        return self.lib.sdp_pipeline_graph_error(self.handle).decode()

    def outputs(self, stream=None):
        """(residual image, model image, components (n, 3), n) as numpy."""
        G = self.G
        res = np.empty(G * G, dtype=np.float32)
        model = np.empty(G * G, dtype=np.float32)
        src = np.zeros((max(1, self.cfg.max_sources), 3), dtype=np.float32)
        n = C.c_int(0)
        check(self.lib.sdp_pipeline_copy_outputs(self.handle, _ptr(res), _ptr(model), _ptr(src), C.byref(n),
                                                 _stream(stream)), self.lib)
        return res, model, src[: max(0, n.value)].copy(), n.value

    def residual_rms(self, stream=None) -> float:
        """FP64 RMS of the last cycle's residual image (on the device)."""
        import torch
        res, model, src, n = _p(), _p(), _p(), _p()
        check(self.lib.sdp_pipeline_outputs(self.handle, C.byref(res), C.byref(model), C.byref(src), C.byref(n)),
              self.lib)
        out = torch.zeros(1, dtype=torch.float64, device=torch.device("cuda", torch.cuda.current_device()))
        check(self.lib.sdp_image_rms(_i(self.G), res, _dp(out), _stream(stream)), self.lib)
        return float(out.item())

    def close(self):
        if self.handle:
            check(self.lib.sdp_pipeline_destroy(self.handle), self.lib)
            self.handle = _p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Device:
    """Device-resident layer over torch CUDA tensors."""

    def __init__(self, lib: C.CDLL | None = None):
        self.lib = lib or load()

    @staticmethod
    def wkernels(kernels, supports_dev, supports_host) -> WKernels:
        sh = np.asarray(supports_host).reshape(-1, 2)
        return WKernels(_dp(kernels), _dp(supports_dev), int(sh.shape[0]), int(kernels.shape[0]),
                        int(sh[:, 0].max()))

    def plan(self, grid_size, oversampling, uv_scale, w_scale, uvw, gk: WKernels, dk: WKernels | None = None,
             mode=SDP_GRID_STD, stream=None, keep=(), options: PlanOptions | None = None) -> VisPlan:
        geom = Geometry(grid_size, oversampling, uv_scale, w_scale)
        return VisPlan(self.lib, geom, gk, dk, uvw, mode, stream, keep, options)

    def autotune(self, grid_size, oversampling, uv_scale, w_scale, uvw, gk: WKernels, dk: WKernels | None,
                 measured, model_grid, residual_grid, degrid_mode=SDP_DEGRID_CONV, reps=3, mode=SDP_GRID_STD,
                 stream=None):
        """Fastest plan shape for this visibility set (sdp_visplan_autotune):
        (PlanOptions, ms per fused pass, shapes timed)."""
        geom = Geometry(grid_size, oversampling, uv_scale, w_scale)
        best = PlanOptions()
        ms = C.c_float(0)
        cand = _i(0)
        dk = dk or gk
        check(self.lib.sdp_visplan_autotune(C.byref(geom), C.byref(gk), C.byref(dk), _i(uvw.shape[0]), _dp(uvw),
                                            _i(mode), _dp(measured), _dp(model_grid), _dp(residual_grid),
                                            _i(degrid_mode), _i(reps), C.byref(best), C.byref(ms), C.byref(cand),
                                            _stream(stream)), self.lib)
        return best, float(ms.value), cand.value

    def batch(self, plans, stream=None) -> VisBatch:
        return VisBatch(self.lib, plans, stream)

    def pipeline(self, cfg: PipelineConfig, uvw, measured, psf, gk: WKernels, dk: WKernels | None = None,
                 stream=None, keep=()) -> Pipeline:
        return Pipeline(self.lib, cfg, gk, dk, uvw, measured, psf, stream, keep)

    def degrid_nearest(self, grid_size, uv_scale, uvw, grid, out, stream=None):
        check(self.lib.sdp_degrid_nearest(_i(grid_size), _d(uv_scale), _i(uvw.shape[0]), _dp(uvw), _dp(grid),
                                          _dp(out), _stream(stream)), self.lib)

    def correct_to_finegrid(self, grid_size, oversampling, uv_scale, uvw, out, stream=None):
        check(self.lib.sdp_correct_to_finegrid(_i(grid_size), _i(oversampling), _d(uv_scale), _i(uvw.shape[0]),
                                               _dp(uvw), _dp(out), _stream(stream)), self.lib)

    def subtract_vis(self, a, b, out, stream=None):
        check(self.lib.sdp_subtract_vis(_i(a.shape[0]), _dp(a), _dp(b), _dp(out), _stream(stream)), self.lib)

    def fft2d(self, grid_size, x, out, sign, stream=None):
        check(self.lib.sdp_fft2d(_i(grid_size), _dp(x), _dp(out), _i(sign), _stream(stream)), self.lib)

    def fft2d_tc(self, grid_size, x, out, sign, work, stream=None):
        """Tensor-core (BF16 split hi/lo) 2-D FFT, G = 1024 / 2048 / 4096."""
        check(self.lib.sdp_fft2d_tc(_i(grid_size), _dp(x), _dp(out), _i(sign), _dp(work), _stream(stream)),
              self.lib)

    def grid_to_image(self, grid_size, grid, prolate_ext, work, image, stream=None):
        check(self.lib.sdp_grid_to_image(_i(grid_size), _dp(grid), _dp(prolate_ext), _dp(work), _dp(image),
                                         _stream(stream)), self.lib)

    def bin_load_vis(self, path, uvw, vis, stream=None):
        """Loads a visibility file into device tensors uvw [n][3], vis [n][2]
        (pinned staging, asynchronous copies); returns (n, snapped)."""
        n, sn = _ll(0), _i(0)
        check(self.lib.sdp_bin_load_vis(str(path).encode(), _ll(min(uvw.shape[0], vis.shape[0])), _dp(uvw), _dp(vis),
                                        C.byref(n), C.byref(sn), _stream(stream)), self.lib)
        return n.value, bool(sn.value)

    def bin_load_kernels(self, path, supports, samples, stream=None):
        """Loads a kernel-set file into device tensors supports [planes][2]
        (int32) and samples [total][2]; returns (planes, total)."""
        npl, tot = _i(0), _ll(0)
        check(self.lib.sdp_bin_load_kernels(str(path).encode(), _i(supports.shape[0]), _ll(samples.shape[0]),
                                            _dp(supports), _dp(samples), C.byref(npl), C.byref(tot),
                                            _stream(stream)), self.lib)
        return npl.value, tot.value

    def bin_load_image(self, path, image, rows, cols, stream=None):
        r, c = _i(0), _i(0)
        check(self.lib.sdp_bin_load_image(str(path).encode(), _i(rows), _i(cols), _dp(image), C.byref(r), C.byref(c),
                                          _stream(stream)), self.lib)
        return r.value, c.value

    def merge_grids(self, grid_size, slices, grids, out, stream=None):
        """out = sum of `slices` contiguous G^2 grids (merge_gridded_visibilities)."""
        check(self.lib.sdp_merge_grids(_i(grid_size), _i(slices), _dp(grids), _dp(out), _stream(stream)), self.lib)

    def image_to_grid(self, grid_size, image, work, grid, stream=None):
        check(self.lib.sdp_image_to_grid(_i(grid_size), _dp(image), _dp(work), _dp(grid), _stream(stream)),
              self.lib)

    def psf_generate(self, plan: "VisPlan", prolate, psf, stream=None):
        """Dirty PSF of a plan's uv coverage, normalised to peak 1; returns the
        peak before normalisation."""
        import torch
        G = plan.geom.grid_size
        dev = psf.device
        ones = torch.empty((max(plan.n, 1), 2), dtype=torch.float32, device=dev)
        grid = torch.empty((G * G, 2), dtype=torch.float32, device=dev)
        work = torch.empty_like(grid)
        mx = torch.zeros(1, dtype=torch.float64, device=dev)
        check(self.lib.sdp_psf_generate(plan.handle, _dp(prolate), _dp(ones), _dp(grid), _dp(work), _dp(psf),
                                        _dp(mx), _stream(stream)), self.lib)
        return float(mx.item())

    def wkernels_generate(self, half_supports, oversampling, max_w, fov_rad, image_samples=256, stream=None):
        """W-projection tables on the device: (gridding, degridding, supports)."""
        import torch
        planes = len(half_supports)
        hs = (_i * planes)(*[int(h) for h in half_supports])
        total = _i(0)
        check(self.lib.sdp_wkernels_generate_sizes(_i(planes), hs, _i(oversampling), C.byref(total)), self.lib)
        self.lib.sdp_wkernels_generate_scratch_bytes.restype = C.c_size_t
        nscr = self.lib.sdp_wkernels_generate_scratch_bytes(_i(planes), hs, _i(oversampling))
        dev = torch.device("cuda", torch.cuda.current_device())
        gk = torch.empty((total.value, 2), dtype=torch.float32, device=dev)
        dk = torch.empty_like(gk)
        sup = torch.empty((planes, 2), dtype=torch.int32, device=dev)
        scr = torch.empty(nscr, dtype=torch.uint8, device=dev)
        check(self.lib.sdp_wkernels_generate(_i(planes), hs, _i(oversampling), _d(max_w), _d(fov_rad),
                                             _i(image_samples), _dp(gk), _dp(dk), _dp(sup), _dp(scr),
                                             C.c_size_t(nscr), _stream(stream)), self.lib)
        return gk, dk, sup

    def image_rms(self, grid_size, image, stream=None) -> float:
        import torch
        out = torch.zeros(1, dtype=torch.float64, device=image.device)
        check(self.lib.sdp_image_rms(_i(grid_size), _dp(image), _dp(out), _stream(stream)), self.lib)
        return float(out.item())

    def prolate_table(self, grid_size, out, stream=None):
        check(self.lib.sdp_prolate_table(_i(grid_size), _dp(out), _stream(stream)), self.lib)

    def dft(self, sources, uvw, vis, stream=None):
        check(self.lib.sdp_dft(_i(uvw.shape[0]), _i(sources.shape[0]), _dp(sources), _dp(uvw), _dp(vis),
                               _stream(stream)), self.lib)

    def hogbom_workspace_bytes(self, grid_size) -> int:
        b = _sz(0)
        check(self.lib.sdp_hogbom_workspace_bytes(_i(grid_size), C.byref(b)), self.lib)
        return b.value

    def hogbom_noalloc(self, params: CleanParams, residual, psf, model, sources, count, stream=None):
        """sdp_hogbom_noalloc: Hogbom with its scratch in a fixed device array
        (no device allocation; grid_size <= 4096)."""
        check(self.lib.sdp_hogbom_noalloc(C.byref(params), _dp(residual), _dp(psf), _dp(model), _dp(sources),
                                          _dp(count), _stream(stream)), self.lib)

    def hogbom(self, params: CleanParams, residual, psf, model, sources, count, workspace, stream=None):
        check(self.lib.sdp_hogbom(C.byref(params), _dp(residual), _dp(psf), _dp(model), _dp(sources), _dp(count),
                                  _dp(workspace), _sz(workspace.numel() * workspace.element_size()),
                                  _stream(stream)), self.lib)

    # -- learned major cycle ------------------------------------------------------------
    def unet_input_planes(self, grid_size, residual, psf, planes, scale, stream=None):
        """planes (3 G^2): r / s, sign(r) sqrt(|r| / s), psf; scale[0] = s = max |r|."""
        check(self.lib.sdp_unet_input_planes(_i(grid_size), _dp(residual), _dp(psf), _dp(planes), _dp(scale),
                                             _stream(stream)), self.lib)

    def unet_input_planes_window(self, grid_size, window, residual, psf, planes, scale, stream=None):
        """The planes of the centred window^2 part of the image (offset
        (grid_size - window) / 2); scale[0] = max |r| over the whole image."""
        check(self.lib.sdp_unet_input_planes_window(_i(grid_size), _i(window), _dp(residual), _dp(psf), _dp(planes),
                                                    _dp(scale), _stream(stream)), self.lib)

    def select_workspace(self):
        import torch
        b = _sz(0)
        check(self.lib.sdp_select_workspace_bytes(C.byref(b)), self.lib)
        return torch.empty(b.value, dtype=torch.uint8, device=torch.device("cuda", torch.cuda.current_device()))

    def select_components(self, grid_size, cell, proposal, scale, rel_threshold, max_count, comps, count,
                          delta_image, workspace, signed=False, stream=None):
        check(self.lib.sdp_select_components(_i(grid_size), _d(cell), _dp(proposal), _dp(scale),
                                             _i(1 if signed else 0), C.c_float(rel_threshold), _i(max_count),
                                             _dp(comps), _dp(count), _dp(delta_image), _dp(workspace),
                                             _stream(stream)), self.lib)

    def dots(self, a, b, out, stream=None):
        check(self.lib.sdp_dots(C.c_longlong(a.numel()), _dp(a), _dp(b), _dp(out), _stream(stream)), self.lib)

    def axpy_ratio(self, dots, alpha_max, x, y, alpha=None, sign=1.0, stream=None):
        """y += sign * alpha * x, alpha = clamp(dots[0] / dots[1], 0, alpha_max)."""
        check(self.lib.sdp_axpy_ratio(C.c_longlong(x.numel()), _dp(dots), _d(alpha_max), C.c_float(sign), _dp(x),
                                      _dp(y), _dp(alpha), _stream(stream)), self.lib)

    def scale(self, x, factor, stream=None):
        check(self.lib.sdp_scale(C.c_longlong(x.numel()), _dp(x), C.c_float(factor), _stream(stream)), self.lib)

    # ---- gain calibration (device layer) ----
    def gaincal_normal_equations(self, receiver_pairs, measured, predicted, gains, A, Q, flags, stream=None):
        check(self.lib.sdp_gaincal_normal_equations(_i(receiver_pairs.shape[0]), _i(gains.shape[0]), _dp(measured),
                                                    _dp(predicted), _dp(gains), _dp(receiver_pairs), _dp(A), _dp(Q),
                                                    _dp(flags), _stream(stream)), self.lib)

    def svd_workspace_bytes(self, n) -> int:
        b = _sz(0)
        check(self.lib.sdp_svd_workspace_bytes(_i(n), C.byref(b)), self.lib)
        return b.value

    def svd(self, n, A, S, U, VT, workspace, stream=None):
        check(self.lib.sdp_svd(_i(n), _dp(A), _dp(S), _dp(U), _dp(VT), _dp(workspace), _sz(workspace.numel()),
                               _stream(stream)), self.lib)

    def svd_check(self, workspace, stream=None) -> int:
        """Raises when the last sdp_svd's barrier wait gave up; returns its sweeps."""
        sw = _i(0)
        check(self.lib.sdp_svd_check(_dp(workspace), C.byref(sw), _stream(stream)), self.lib)
        return sw.value

    PEAK_KINDS = {"l2_read": 0, "smem_read": 1, "fp32_fma": 2, "fp32x2_fma": 3, "hogbom_update": 4}

    def peak(self, kind: str, scratch, reps: int = 10, stream=None) -> float:
        """Measured on-chip ceiling (sdp_peak_measure): bytes/s for l2_read and
        smem_read, FLOP/s for the FMA kinds, pixel updates/s for hogbom_update.
        scratch: a device tensor (its size is the L2 read buffer)."""
        r = C.c_double(0.0)
        check(self.lib.sdp_peak_measure(_i(self.PEAK_KINDS[kind]), _dp(scratch),
                                        _sz(scratch.numel() * scratch.element_size()), _i(reps), C.byref(r),
                                        _stream(stream)), self.lib)
        return r.value

    def gaincal_suq(self, n, S, U, Q, SUQ, stream=None):
        check(self.lib.sdp_gaincal_suq(_i(n), _dp(S), _dp(U), _dp(Q), _dp(SUQ), _stream(stream)), self.lib)

    def gaincal_update(self, n, SUQ, VT, gains_in, gains_out, stream=None):
        check(self.lib.sdp_gaincal_update(_i(n), _i(gains_in.shape[0]), _dp(SUQ), _dp(VT), _dp(gains_in),
                                          _dp(gains_out), _stream(stream)), self.lib)

    def zero_border(self, grid_size, border, image, stream=None):
        check(self.lib.sdp_zero_border(_i(grid_size), _i(border), _dp(image), _stream(stream)), self.lib)

    def sky_render(self, grid_size, cell, comps, image, stream=None):
        check(self.lib.sdp_sky_render(_i(grid_size), _d(cell), _i(comps.shape[0]), _dp(comps), _dp(image),
                                      _stream(stream)), self.lib)

    def dft_gauss(self, sources, uvw, vis, stream=None):
        check(self.lib.sdp_dft_gauss(_i(uvw.shape[0]), _i(sources.shape[0]), _dp(sources), _dp(uvw), _dp(vis),
                                     _stream(stream)), self.lib)

    def dft_pixels(self, comps, cell, uvw, vis, accumulate=False, stream=None):
        """comps [k][3 or 4] (l, m, flux[, ...]) on the pixel grid of cell."""
        check(self.lib.sdp_dft_pixels(_i(uvw.shape[0]), _i(comps.shape[0]), _dp(comps), _i(comps.shape[1]),
                                      _d(cell), _dp(uvw), _dp(vis), _i(1 if accumulate else 0), _stream(stream)),
              self.lib)

    def add_vis(self, a, b, out, stream=None):
        check(self.lib.sdp_add_vis(_i(a.shape[0]), _dp(a), _dp(b), _dp(out), _stream(stream)), self.lib)

    def blur_mse(self, pred, target, scratch, grad, loss, stream=None):
        """loss[0] (device double) = mean((b * (pred - target))^2); grad = d loss / d pred
        (may be None); pred/target [n][h][w]; scratch 2 n h w floats."""
        n, h, w = pred.shape
        check(self.lib.sdp_blur_mse(_i(n), _i(h), _i(w), _dp(pred), _dp(target), _dp(scratch), _dp(grad),
                                    _dp(loss), _stream(stream)), self.lib)


class UNet:
    """The learned-proposal U-Net on the device (sdp_unet_*): 4 levels, base
    32 channels, BF16 weights and activations with FP32 accumulation."""

    def __init__(self, lib, in_channels: int, max_batch: int, max_height: int, max_width: int,
                 training: bool = True, base: int = 32):
        self.lib = lib
        self.in_channels = in_channels
        self.handle = _p()
        check(lib.sdp_unet_create(C.byref(self.handle), _i(base), _i(in_channels), _i(max_batch), _i(max_height),
                                  _i(max_width), _i(1 if training else 0)), lib)
        n = _sz(0)
        check(lib.sdp_unet_num_params(self.handle, C.byref(n)), lib)
        self.num_params = n.value

    def close(self):
        if self.handle:
            check(self.lib.sdp_unet_destroy(self.handle), self.lib)
            self.handle = _p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def layer(self, k: int):
        ci, co, wo, bo = _i(0), _i(0), _sz(0), _sz(0)
        check(self.lib.sdp_unet_layer(self.handle, _i(k), C.byref(ci), C.byref(co), C.byref(wo), C.byref(bo)),
              self.lib)
        return ci.value, co.value, wo.value, bo.value

    def set_params(self, params, stream=None):
        """params: float32 numpy array (host) or CUDA tensor of num_params."""
        if isinstance(params, np.ndarray):
            a = np.ascontiguousarray(params, dtype=np.float32)
            assert a.size == self.num_params
            check(self.lib.sdp_unet_set_params(self.handle, a.ctypes.data_as(_p), _stream(stream)), self.lib)
            import torch
            torch.cuda.synchronize()  # the host array may go away
        else:
            assert params.numel() == self.num_params
            check(self.lib.sdp_unet_set_params(self.handle, _dp(params), _stream(stream)), self.lib)

    def get_params(self, stream=None) -> np.ndarray:
        import torch
        out = np.empty(self.num_params, np.float32)
        check(self.lib.sdp_unet_get_params(self.handle, out.ctypes.data_as(_p), _stream(stream)), self.lib)
        torch.cuda.synchronize()
        return out

    def get_grads(self, stream=None) -> np.ndarray:
        import torch
        out = np.empty(self.num_params, np.float32)
        check(self.lib.sdp_unet_get_grads(self.handle, out.ctypes.data_as(_p), _stream(stream)), self.lib)
        torch.cuda.synchronize()
        return out

    def zero_grads(self, stream=None):
        check(self.lib.sdp_unet_zero_grads(self.handle, _stream(stream)), self.lib)

    def forward(self, x, out, scale=None, stream=None):
        """x [n][in_channels][h][w] -> out [n][h][w] (CUDA float32 tensors)."""
        n, c, h, w = x.shape
        assert c == self.in_channels
        check(self.lib.sdp_unet_forward(self.handle, _i(n), _i(h), _i(w), _dp(x), _dp(scale), _dp(out),
                                        _stream(stream)), self.lib)

    def backward(self, grad_out, stream=None):
        check(self.lib.sdp_unet_backward(self.handle, _dp(grad_out), _stream(stream)), self.lib)

    def set_tensor_path(self, tcgen05: bool):
        check(self.lib.sdp_unet_set_tensor_path(self.handle, _i(1 if tcgen05 else 0)), self.lib)

    def check(self, stream=None):
        """Raises when a tensor-core convolution gave up a bounded wait."""
        check(self.lib.sdp_unet_check(self.handle, _stream(stream)), self.lib)

    def set_wait_limit(self, epilogue_polls: int):
        """Polls of the tensor-core epilogue's bounded wait (0: the default);
        a tiny value makes the wait run out (the failure path)."""
        check(self.lib.sdp_unet_set_wait_limit(self.handle, C.c_longlong(epilogue_polls)), self.lib)

    def adam_step(self, lr, beta1=0.9, beta2=0.999, eps=1e-8, stream=None):
        check(self.lib.sdp_unet_adam_step(self.handle, C.c_float(lr), C.c_float(beta1), C.c_float(beta2),
                                          C.c_float(eps), _stream(stream)), self.lib)
