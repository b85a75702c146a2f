"""Binary input files (sdp_bin_*): no counterpart in the reference, which
reads text files (top.c:139-222, 224-380, 453-510).

* host round trips of visibilities, kernel sets and images are bit-exact,
  including empty files and sizes that are not multiples of the staging
  chunk;
* visibilities parsed by the CSV set-up actor (visibility_host_set_up,
  bit-exact with the reference in test_loaders) and written to a binary
  file come back identical;
* corrupt, truncated or mismatched files are refused with SDP_ERR_DATA, a
  missing file with SDP_ERR_IO, buffers that are too small with
  SDP_ERR_RANGE;
* (GPU) the device loads, through pinned staging and asynchronous copies,
  equal the host arrays bit for bit, for a file larger than the staging ring.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import test_loaders as TL

_i, _p = C.c_int, C.c_void_p


@pytest.fixture(scope="module")
def lib(sdp):
    return sdp.load()


@pytest.mark.parametrize("n", [0, 1, 12_345, 1_000_003])
def test_vis_round_trip(sdp, lib, tmp_path, n):
    rng = np.random.default_rng(n)
    uvw = rng.standard_normal((n, 3)).astype(np.float32)
    vis = rng.standard_normal((n, 2)).astype(np.float32)
    f = tmp_path / "v.bin"
    sdp.bin_write_vis(f, uvw, vis, snapped=(n % 2 == 1))
    assert sdp.bin_info(f) == (1, n, n % 2)
    u, v, sn = sdp.bin_read_vis_host(f)
    np.testing.assert_array_equal(u, uvw)
    np.testing.assert_array_equal(v, vis)
    assert sn == (n % 2 == 1)


def test_kernels_and_image_headers(sdp, tmp_path):
    sup = np.array([[4, 0], [3, 6400]], np.int32)
    k = np.random.default_rng(1).standard_normal((6400 + 4096, 2)).astype(np.float32)
    sdp.bin_write_kernels(tmp_path / "k.bin", sup, k)
    assert sdp.bin_info(tmp_path / "k.bin") == (2, k.shape[0], 2)
    img = np.random.default_rng(2).standard_normal((33, 65)).astype(np.float32)
    sdp.bin_write_image(tmp_path / "i.bin", img)
    assert sdp.bin_info(tmp_path / "i.bin") == (3, 33, 65)


def test_csv_to_binary_is_exact(sdp, lib, tmp_path):
    rng = np.random.default_rng(9)
    path = tmp_path / "vis.csv"
    TL._vis_file(path, rng, 3000, 3000)
    cfg, keep = TL._cfg(tmp_path, visibility_source_file=str(path), frequency_hz=1.4e8, right_ascension=True,
                        force_weight_to_one=True, max_w=1500.0)
    uvw = np.zeros((3000, 3), np.float32)
    vis = np.zeros((3000, 2), np.float32)
    lib.visibility_host_set_up(_i(3000), C.byref(cfg), uvw.ctypes.data_as(_p), vis.ctypes.data_as(_p))
    assert lib.sdp_last_status() == 0
    sdp.bin_write_vis(tmp_path / "vis.bin", uvw, vis)
    u, v, _ = sdp.bin_read_vis_host(tmp_path / "vis.bin")
    np.testing.assert_array_equal(u, uvw)
    np.testing.assert_array_equal(v, vis)


def test_bad_files_refused(sdp, lib, tmp_path):
    with pytest.raises(sdp.SdpError) as e:
        sdp.bin_info(tmp_path / "missing.bin")
    assert e.value.status == sdp.SDP_ERR_IO
    (tmp_path / "junk.bin").write_bytes(b"not a binary file at all" * 10)
    with pytest.raises(sdp.SdpError) as e:
        sdp.bin_info(tmp_path / "junk.bin")
    assert e.value.status == sdp.SDP_ERR_DATA
    uvw = np.zeros((1000, 3), np.float32)
    vis = np.zeros((1000, 2), np.float32)
    f = tmp_path / "v.bin"
    sdp.bin_write_vis(f, uvw, vis)
    data = f.read_bytes()
    (tmp_path / "short.bin").write_bytes(data[:-100])
    with pytest.raises(sdp.SdpError) as e:
        sdp.bin_read_vis_host(tmp_path / "short.bin")
    assert e.value.status == sdp.SDP_ERR_DATA
    sdp.bin_write_image(tmp_path / "i.bin", np.zeros((4, 4), np.float32))
    with pytest.raises(sdp.SdpError) as e:
        sdp.bin_read_vis_host(tmp_path / "i.bin")
    assert e.value.status == sdp.SDP_ERR_DATA
    lib.sdp_clear_error()  # the status is thread-local and outlives the call


@pytest.mark.gpu
def test_device_loads_exact(sdp, device, tmp_path):
    import torch
    rng = np.random.default_rng(4)
    n = 9_000_001  # 108 MB of uvw: more than the 4 x 32 MB staging ring
    uvw = rng.standard_normal((n, 3)).astype(np.float32)
    vis = rng.standard_normal((n, 2)).astype(np.float32)
    sdp.bin_write_vis(tmp_path / "v.bin", uvw, vis, snapped=True)
    ud = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    vd = torch.empty((n, 2), dtype=torch.float32, device="cuda")
    got, sn = device.bin_load_vis(tmp_path / "v.bin", ud, vd)
    assert got == n and sn
    np.testing.assert_array_equal(ud.cpu().numpy(), uvw)
    np.testing.assert_array_equal(vd.cpu().numpy(), vis)
    with pytest.raises(sdp.SdpError) as e:
        device.bin_load_vis(tmp_path / "v.bin", ud[:10], vd[:10])
    assert e.value.status == sdp.SDP_ERR_RANGE
    sup = np.array([[4, 0], [3, 6400]], np.int32)
    k = rng.standard_normal((6400 + 4096, 2)).astype(np.float32)
    sdp.bin_write_kernels(tmp_path / "k.bin", sup, k)
    sd = torch.empty((4, 2), dtype=torch.int32, device="cuda")
    kd = torch.empty((20000, 2), dtype=torch.float32, device="cuda")
    assert device.bin_load_kernels(tmp_path / "k.bin", sd, kd) == (2, k.shape[0])
    np.testing.assert_array_equal(sd[:2].cpu().numpy(), sup)
    np.testing.assert_array_equal(kd[:k.shape[0]].cpu().numpy(), k)
    img = rng.standard_normal((2048, 2048)).astype(np.float32)
    sdp.bin_write_image(tmp_path / "p.bin", img)
    idev = torch.empty(2048 * 2048, dtype=torch.float32, device="cuda")
    assert device.bin_load_image(tmp_path / "p.bin", idev, 2048, 2048) == (2048, 2048)
    np.testing.assert_array_equal(idev.cpu().numpy().reshape(2048, 2048), img)
