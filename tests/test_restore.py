"""Restoring and writing (major_loop_iter.c:8-46, 168-278).

* conv2D (model * clean-PSF window) on the GPU against the reference's own
  conv2D compiled from its sources: bit-exact, including negative and
  below-threshold model pixels (skipped), the 1e-5 threshold itself (in
  double, as the reference compares) and a NaN pixel (it contributes);
* save_output / save_extracted_sources_actor: the files they write equal the
  reference's byte for byte;
* save_image_to_file (host only): the "%f, " text of the reference.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle as O

_i, _p = C.c_int, C.c_void_p


class Int2(C.Structure):
    _fields_ = [("x", C.c_int), ("y", C.c_int)]


def _ref():
    if not O.RefLib.available("f32"):
        pytest.skip("reference build oracle/_ref not present")
    return O.RefLib("f32").lib


def _model(G, rng):
    m = np.zeros(G * G, np.float32)
    idx = rng.choice(G * G, 300, replace=False)
    m[idx] = rng.standard_normal(300).astype(np.float32)  # half negative: skipped
    m[idx[:5]] = np.float32(1e-5)                          # below 1e-5 in double
    m[idx[5:8]] = np.nextafter(np.float32(1e-5), np.float32(1))
    m[idx[8]] = np.nan
    m[0] = 2.0                                            # corner: window clipped
    m[G * G - 1] = 3.0
    return m


def _psf(G):
    y, x = np.mgrid[0:G, 0:G]
    c = G // 2
    return np.exp(-((x - c) ** 2 / 18.0 + (y - c) ** 2 / 11.0)).astype(np.float32).reshape(-1)


@pytest.mark.gpu
@pytest.mark.parametrize("G,hx,hy", [(256, 12, 9), (128, 3, 20), (64, 1, 1)])
def test_conv2d_bit_exact(sdp, G, hx, hy):
    lib = sdp.load()
    ref = _ref()
    rng = np.random.default_rng(G + hx)
    model, psf = _model(G, rng), _psf(G)
    out = np.empty(G * G, np.float32)
    lib.sdp_clear_error()
    lib.conv2D(model.ctypes.data_as(_p), psf.ctypes.data_as(_p), out.ctypes.data_as(_p), _i(G), Int2(hx, hy))
    assert lib.sdp_last_status() == 0, lib.sdp_last_error()
    exp = np.empty_like(out)
    ref.conv2D(model.ctypes.data_as(_p), psf.ctypes.data_as(_p), exp.ctypes.data_as(_p), _i(G), Int2(hx, hy))
    np.testing.assert_array_equal(out, exp)


def _cfg(tmp_path, tag):
    c = O.make_config(64, 1.0, 1.0, 8)
    keep = []
    for name in ("output_path", "residual_image_output", "psf_image_output", "clean_psf_image_output",
                 "model_image_output", "final_image_output", "model_sources_output"):
        val = str(tmp_path / tag) + "/" if name == "output_path" else name + ".csv"
        b = C.create_string_buffer(val.encode())
        keep.append(b)
        setattr(c, name, C.cast(b, _p))
    (tmp_path / tag).mkdir(exist_ok=True)
    return c, keep


@pytest.mark.gpu
def test_save_output_files_match_reference(sdp, tmp_path):
    lib = sdp.load()
    ref = _ref()
    G = 128
    rng = np.random.default_rng(2)
    res = (rng.standard_normal(G * G) * 1e-3).astype(np.float32)
    model, psf = _model(G, rng), _psf(G)
    clean = _psf(G)
    half = Int2(6, 5)
    cyc = C.c_int(3)
    lib.sdp_clear_error()
    for tag, l in (("b200", lib), ("ref", ref)):
        cfg, keep = _cfg(tmp_path, tag)
        l.save_output(_i(G), res.ctypes.data_as(_p), model.ctypes.data_as(_p), clean.ctypes.data_as(_p), C.byref(half),
                      psf.ctypes.data_as(_p), C.byref(cfg), C.byref(cyc))
        src = np.array([[0.0, 0.0, 1.5], [3e-4, -2e-4, 0.25]], np.float32)
        ns = C.c_int(2)
        img_out = np.empty(G * G, np.float32)
        cfg.cell_size = 1e-4
        l.save_extracted_sources_actor(_i(G), _i(1), _i(2), C.byref(ns), src.ctypes.data_as(_p), C.byref(cyc),
                                       C.byref(cfg), res.ctypes.data_as(_p), clean.ctypes.data_as(_p), C.byref(half),
                                       img_out.ctypes.data_as(_p))
    assert lib.sdp_last_status() == 0, lib.sdp_last_error()
    names = sorted(p.name for p in (tmp_path / "ref").iterdir())
    assert len(names) == 6
    for n in names:
        assert (tmp_path / "b200" / n).read_bytes() == (tmp_path / "ref" / n).read_bytes(), n


def test_save_image_to_file_text(sdp, tmp_path):
    lib = sdp.load()
    rng = np.random.default_rng(8)
    img = (rng.standard_normal(300 * 300) * 10.0 ** rng.integers(-8, 8, 300 * 300)).astype(np.float32)
    img[:3] = [np.inf, -0.0, 1e30]
    outs = []
    libs = [("b200", lib)] + ([("ref", O.RefLib("f32").lib)] if O.RefLib.available("f32") else [])
    for tag, l in libs:
        cfg, keep = _cfg(tmp_path, tag)
        name = C.create_string_buffer(b"img.csv")
        l.save_image_to_file(C.byref(cfg), img.ctypes.data_as(_p), name, _i(0), _i(0), _i(300), _i(300), _i(1))
        outs.append((tmp_path / tag / "cycle_1_img.csv").read_bytes())
    expected = "".join("".join("%f, " % float(v) for v in img[r * 300:(r + 1) * 300]) + "\n"
                       for r in range(300)).encode()
    for o in outs:
        assert o == expected
