"""File-reading set-up actors (top.c:139-380, 453-510) against the reference.

The library's multi-threaded parsers must give the reference's arrays bit
for bit: the same float rounding of every value, the RA flip, weights, the
w clamp (with the float build's fabsf), the kernel-support offsets, the PSF
crop and its maximum, and fscanf's behaviour on short files (stale values
keep being transformed).  Compared with the reference's own set-up code
compiled from its sources (oracle/_ref) where it is built, and always with
a numpy restatement of the same arithmetic.  No GPU is used.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle as O

_i, _d, _p = C.c_int, C.c_double, C.c_void_p


@pytest.fixture(scope="module")
def lib(sdp):
    return sdp.load()


def _fmt(rng, x):
    k = rng.integers(0, 5)
    if k == 0:
        return f"{x:.17g}"
    if k == 1:
        return f"{x:e}"
    if k == 2:
        return f"+{x:.9f}" if x >= 0 else f"{x:.9f}"
    if k == 3:
        return f"{x:.3E}"
    return f"{x:.6f}"


def _vis_file(path, rng, n_rec, declared, partial=0):
    rows = rng.standard_normal((n_rec, 6)) * np.array([900.0, 900.0, 60.0, 1.0, 1.0, 0.4]) + \
        np.array([0, 0, 0, 0, 0, 1.0])
    rows[::7, 2] *= 40.0  # beyond max_w
    lines = [str(declared)]
    for r in rows:
        lines.append(" ".join(_fmt(rng, v) for v in r))
    if partial:
        lines.append(" ".join(_fmt(rng, v) for v in rng.standard_normal(partial)))
    path.write_text("\n".join(lines) + "\n")
    return rows


def _cfg(tmp_path, **kw):
    c = O.make_config(64, 1.0, 1.0, 8)
    keep = []
    for name, val in kw.items():
        if isinstance(val, str):
            b = C.create_string_buffer(val.encode())
            keep.append(b)
            setattr(c, name, C.cast(b, _p))
        else:
            setattr(c, name, val)
    return c, keep


def _vis_restated(t, n, freq, ra, w1, max_w):
    """top.c:171-219 over the parsed numbers t (stale fields once t ends)."""
    m2w = freq / 299792458.0
    f = [0.0] * 6
    uvw = np.zeros((n, 3), np.float32)
    vis = np.zeros((n, 2), np.float32)
    for i in range(n):
        for k in range(6):
            if 6 * i + k < len(t):
                f[k] = t[6 * i + k]
        if ra:
            f[0] *= -1.0
            f[2] *= -1.0
        if not w1:
            f[3] *= f[5]
            f[4] *= f[5]
        aw = float(abs(np.float32(f[2])))
        if aw > max_w:
            f[2] = f[2] / aw * max_w
        uvw[i] = [np.float32(f[0] * m2w), np.float32(f[1] * m2w), np.float32(f[2] * m2w)]
        vis[i] = [np.float32(f[3]), np.float32(f[4])]
    return uvw, vis


@pytest.mark.parametrize("ra,w1,n_rec,declared,partial", [(True, True, 2000, 2000, 0), (False, False, 2000, 2000, 0),
                                                          (True, False, 300, 310, 4)])
def test_visibility_host_set_up(lib, tmp_path, ra, w1, n_rec, declared, partial):
    rng = np.random.default_rng(n_rec + partial)
    path = tmp_path / "vis.csv"
    _vis_file(path, rng, n_rec, declared, partial)
    cfg, keep = _cfg(tmp_path, visibility_source_file=str(path), frequency_hz=1.4e8, right_ascension=ra,
                     force_weight_to_one=w1, max_w=1500.0)
    uvw = np.zeros((declared, 3), np.float32)
    vis = np.zeros((declared, 2), np.float32)
    lib.sdp_clear_error()
    lib.visibility_host_set_up(_i(declared), C.byref(cfg), uvw.ctypes.data_as(_p), vis.ctypes.data_as(_p))
    assert lib.sdp_last_status() == 0
    toks = path.read_text().split()[1:]
    t = [float(x) for x in toks]
    eu, ev = _vis_restated(t, declared, 1.4e8, ra, w1, 1500.0)
    np.testing.assert_array_equal(uvw, eu)
    np.testing.assert_array_equal(vis, ev)
    if O.RefLib.available("f32"):
        r = O.RefLib("f32").lib
        ru = np.zeros_like(uvw)
        rv = np.zeros_like(vis)
        r.visibility_host_set_up(_i(declared), C.byref(cfg), ru.ctypes.data_as(_p), rv.ctypes.data_as(_p))
        np.testing.assert_array_equal(uvw, ru)
        np.testing.assert_array_equal(vis, rv)


def test_kernel_host_set_up(lib, tmp_path):
    rng = np.random.default_rng(5)
    OS, hs = 8, [2, 3, 1, 4]
    ns = [((h + 1) * OS) ** 2 for h in hs]
    (tmp_path / "sup.txt").write_text("\n".join(map(str, hs)) + "\n")
    re_v = rng.standard_normal(sum(ns))
    im_v = rng.standard_normal(sum(ns) - 17)  # short imaginary file: the tail reads 0.0
    (tmp_path / "re.txt").write_text(" ".join(_fmt(rng, v) for v in re_v))
    (tmp_path / "im.txt").write_text("\n".join(_fmt(rng, v) for v in im_v))
    files = dict(kernel_support_file=str(tmp_path / "sup.txt"), kernel_real_file=str(tmp_path / "re.txt"),
                 kernel_imag_file=str(tmp_path / "im.txt"), degridding_kernel_support_file=str(tmp_path / "sup.txt"),
                 degridding_kernel_real_file=str(tmp_path / "im.txt"),
                 degridding_kernel_imag_file=str(tmp_path / "re.txt"))
    cfg, keep = _cfg(tmp_path, oversampling=OS, **files)
    for fn in ("kernel_host_set_up", "degridding_kernel_host_set_up"):
        sup = np.zeros((4, 2), np.int32)
        k = np.zeros((sum(ns), 2), np.float32)
        getattr(lib, fn)(_i(4), _i(sum(ns)), C.byref(cfg), sup.ctypes.data_as(_p), k.ctypes.data_as(_p))
        assert lib.sdp_last_status() == 0
        np.testing.assert_array_equal(sup[:, 0], hs)
        np.testing.assert_array_equal(sup[:, 1], np.concatenate([[0], np.cumsum(ns)[:-1]]))
        re_t = np.float32([float(x) for x in (tmp_path / "re.txt").read_text().split()])
        im_t = np.concatenate([np.float32([float(x) for x in (tmp_path / "im.txt").read_text().split()]),
                               np.zeros(17, np.float32)])
        exp_re, exp_im = (re_t, im_t) if fn == "kernel_host_set_up" else (im_t, re_t)
        np.testing.assert_array_equal(k[:, 0], exp_re)
        np.testing.assert_array_equal(k[:, 1], exp_im)
        if O.RefLib.available("f32"):
            r = O.RefLib("f32").lib
            rs = np.zeros_like(sup)
            rk = np.zeros_like(k)
            getattr(r, fn)(_i(4), _i(sum(ns)), C.byref(cfg), rs.ctypes.data_as(_p), rk.ctypes.data_as(_p))
            np.testing.assert_array_equal(sup, rs)
            np.testing.assert_array_equal(k, rk)


@pytest.mark.parametrize("G,PG,short", [(64, 96, 0), (128, 96, 0), (64, 64, 100)])
def test_psf_host_set_up(lib, tmp_path, G, PG, short):
    rng = np.random.default_rng(G + PG)
    n = PG * PG - short
    vals = np.abs(rng.standard_normal(n)) * 3.0
    (tmp_path / "psf.txt").write_text(" ".join(_fmt(rng, v) for v in vals))
    cfg, keep = _cfg(tmp_path, psf_input_file=str(tmp_path / "psf.txt"))
    psf = np.full(G * G, 9.0, np.float32)
    mx = C.c_double(0.0)
    lib.psf_host_set_up(_i(G), _i(PG), C.byref(cfg), psf.ctypes.data_as(_p), C.byref(mx))
    assert lib.sdp_last_status() == 0
    t = [float(x) for x in (tmp_path / "psf.txt").read_text().split()]
    full = np.zeros(PG * PG, np.float32)
    m = 0.0
    s = 0.0
    for i in range(PG * PG):
        if i < len(t):
            s = t[i]
        full[i] = np.float32(s)
        if s > m:
            m = float(np.float32(s))
    assert mx.value == m
    exp = np.zeros(G * G, np.float32)
    sm, po, go = min(PG, G), max(0, (PG - G) // 2), max(0, (G - PG) // 2)
    for y in range(sm):
        exp[(y + go) * G + go:(y + go) * G + go + sm] = full[(y + po) * PG + po:(y + po) * PG + po + sm]
    exp = (exp.astype(np.float64) / m).astype(np.float32)
    np.testing.assert_array_equal(psf, exp)
    if O.RefLib.available("f32"):
        r = O.RefLib("f32").lib
        rp = np.zeros_like(psf)
        rm = C.c_double(0.0)
        r.psf_host_set_up(_i(G), _i(PG), C.byref(cfg), rp.ctypes.data_as(_p), C.byref(rm))
        assert rm.value == mx.value
        np.testing.assert_array_equal(psf, rp)


def test_count_token_with_fraction(lib, tmp_path):
    """fscanf("%d") takes the digits of "3.25"; the first "%lf" then reads ".25"."""
    (tmp_path / "v.csv").write_text("3.25 1 2 3 4 5\n6 7 8 9 10 11 12\n")
    cfg, keep = _cfg(tmp_path, visibility_source_file=str(tmp_path / "v.csv"), frequency_hz=299792458.0,
                     right_ascension=False, force_weight_to_one=True, max_w=1e9)
    uvw = np.zeros((2, 3), np.float32)
    vis = np.zeros((2, 2), np.float32)
    lib.visibility_host_set_up(_i(2), C.byref(cfg), uvw.ctypes.data_as(_p), vis.ctypes.data_as(_p))
    np.testing.assert_array_equal(uvw, [[0.25, 1, 2], [6, 7, 8]])
    np.testing.assert_array_equal(vis, [[3, 4], [9, 10]])
    if O.RefLib.available("f32"):
        r = O.RefLib("f32").lib
        ru, rv = np.zeros_like(uvw), np.zeros_like(vis)
        r.visibility_host_set_up(_i(2), C.byref(cfg), ru.ctypes.data_as(_p), rv.ctypes.data_as(_p))
        np.testing.assert_array_equal(uvw, ru)
        np.testing.assert_array_equal(vis, rv)


def test_missing_file_sets_io_error(lib, tmp_path):
    cfg, keep = _cfg(tmp_path, visibility_source_file=str(tmp_path / "absent.csv"), frequency_hz=1.4e8)
    uvw = np.zeros((4, 3), np.float32)
    vis = np.zeros((4, 2), np.float32)
    lib.sdp_clear_error()
    lib.visibility_host_set_up(_i(4), C.byref(cfg), uvw.ctypes.data_as(_p), vis.ctypes.data_as(_p))
    assert lib.sdp_last_status() == 7
