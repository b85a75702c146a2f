"""Measured on-chip ceilings (sdp_peak_measure): argument checks on the CPU;
on the GPU every kind returns a rate inside the B200's plausible range, and
the L2 read rate of a buffer that stays on chip is above the HBM copy rate
measured by a plain device-to-device copy of a buffer four times L2's size."""
from __future__ import annotations

import ctypes as C

import pytest


def test_peak_argument_checks(sdp):
    lib = sdp.load()
    r = C.c_double(0.0)
    assert lib.sdp_peak_measure(C.c_int(99), C.c_void_p(16), C.c_size_t(1 << 20), C.c_int(1), C.byref(r),
                                None) == sdp.SDP_ERR_INVALID
    assert lib.sdp_peak_measure(C.c_int(0), None, C.c_size_t(1 << 20), C.c_int(1), C.byref(r),
                                None) == sdp.SDP_ERR_INVALID
    assert lib.sdp_peak_measure(C.c_int(0), C.c_void_p(16), C.c_size_t(1024), C.c_int(1), C.byref(r),
                                None) == sdp.SDP_ERR_INVALID
    assert lib.sdp_peak_measure(C.c_int(0), C.c_void_p(16), C.c_size_t(1 << 20), C.c_int(0), C.byref(r),
                                None) == sdp.SDP_ERR_INVALID
    lib.sdp_clear_error()


@pytest.mark.gpu
def test_peaks_in_plausible_range(sdp):
    import torch
    D = sdp.Device(sdp.load())
    scratch = torch.zeros(32 << 20, dtype=torch.uint8, device="cuda")
    bounds = {"l2_read": (2e12, 1e14), "smem_read": (1e13, 1e15), "fp32_fma": (2e13, 3e14),
              "fp32x2_fma": (2e13, 6e14), "hogbom_update": (1e10, 1e13)}
    got = {k: D.peak(k, scratch, reps=5) for k in bounds}
    for k, (lo, hi) in bounds.items():
        assert lo < got[k] < hi, (k, got[k])
    # HBM: device-to-device copy of 512 MB (read + write bytes)
    a = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    b = torch.empty_like(a)
    b.copy_(a)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(3):
        b.copy_(a)
    e1.record()
    torch.cuda.synchronize()
    hbm = 3 * 2 * a.numel() / (e0.elapsed_time(e1) * 1e-3)
    assert got["l2_read"] > hbm, (got["l2_read"], hbm)
