"""Gains (gains_apply_run.c:4-120, top.c:71-136) against the reference.

Receiver pairs, unit / file gains, the gain reciprocal and the per-visibility
gain products (with and without the subtraction of a prediction) equal the
reference's compiled code bit for bit (oracle/_ref), with random complex
gains and baseline-major indexing over several time steps.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle as O

_i, _p = C.c_int, C.c_void_p
NRX = 24
NBL = NRX * (NRX - 1) // 2
NV = NBL * 7


def _ref():
    if not O.RefLib.available("f32"):
        pytest.skip("reference build oracle/_ref not present")
    return O.RefLib("f32").lib


def _pairs(lib):
    p = np.zeros((NBL, 2), np.int32)
    lib.calculate_receiver_pairs(_i(NBL), _i(NRX), p.ctypes.data_as(_p))
    return p


def test_receiver_pairs_and_gains_file(sdp, tmp_path):
    lib = sdp.load()
    p = _pairs(lib)
    exp = [(a, b) for a in range(NRX) for b in range(a + 1, NRX)]
    np.testing.assert_array_equal(p, exp)
    rng = np.random.default_rng(1)
    g = rng.standard_normal((NRX - 3, 2))  # a short file: the last values repeat
    path = tmp_path / "gains.txt"
    path.write_text("\n".join(f"{a:.12g} {b:.12g}" for a, b in g))
    cfg = O.make_config(64, 1.0, 1.0, 8)
    buf = C.create_string_buffer(str(path).encode())
    cfg.default_gains_file = C.cast(buf, _p)
    libs = [lib] + ([O.RefLib("f32").lib] if O.RefLib.available("f32") else [])
    outs = []
    for use_default in (True, False):
        cfg.use_default_gains = use_default
        for l in libs:
            gains = np.zeros((NRX, 2), np.float32)
            pairs = np.zeros((NBL, 2), np.int32)
            l.gains_host_set_up(_i(NRX), _i(NBL), C.byref(cfg), gains.ctypes.data_as(_p), pairs.ctypes.data_as(_p))
            outs.append((use_default, gains, pairs))
    for use_default, gains, pairs in outs:
        np.testing.assert_array_equal(pairs, exp)
        if use_default:
            np.testing.assert_array_equal(gains, np.tile([1.0, 0.0], (NRX, 1)))
        else:
            np.testing.assert_array_equal(gains[:NRX - 3], g.astype(np.float32))
            np.testing.assert_array_equal(gains[NRX - 3:], np.tile(g[-1].astype(np.float32), (3, 1)))


@pytest.mark.gpu
def test_reciprocal_and_apply_bit_exact(sdp):
    lib = sdp.load()
    ref = _ref()
    rng = np.random.default_rng(2)
    gains = (rng.standard_normal((NRX, 2)) * 0.3 + np.array([1.0, 0.0])).astype(np.float32)
    meas = rng.standard_normal((NV, 2)).astype(np.float32)
    pred = rng.standard_normal((NV, 2)).astype(np.float32)
    pairs = _pairs(lib)
    cfg = O.make_config(64, 1.0, 1.0, 8)
    lib.sdp_clear_error()
    rec, rrec = np.zeros_like(gains), np.zeros_like(gains)
    lib.reciprocal_transform_actor(_i(NRX), gains.ctypes.data_as(_p), C.byref(cfg), rec.ctypes.data_as(_p))
    ref.reciprocal_transform_actor(_i(NRX), gains.ctypes.data_as(_p), C.byref(cfg), rrec.ctypes.data_as(_p))
    np.testing.assert_array_equal(rec, rrec)
    for name, args in (("apply_gains_actor", (0,)), ("apply_gains_actor", (1,)), ("subtract_from_measurements", ())):
        out, rout = np.zeros_like(meas), np.zeros_like(meas)
        for l, o in ((lib, out), (ref, rout)):
            getattr(l, name)(*[_i(a) for a in args], _i(NRX), _i(NBL), _i(NV), meas.ctypes.data_as(_p),
                             pred.ctypes.data_as(_p), rec.ctypes.data_as(_p), pairs.ctypes.data_as(_p), C.byref(cfg),
                             o.ctypes.data_as(_p))
        np.testing.assert_array_equal(out, rout)
    out, rout = np.zeros_like(meas), np.zeros_like(meas)
    for l, o in ((lib, out), (ref, rout)):
        l.apply_gains_only(_i(NRX), _i(NBL), _i(NV), meas.ctypes.data_as(_p), rec.ctypes.data_as(_p),
                           pairs.ctypes.data_as(_p), C.byref(cfg), o.ctypes.data_as(_p))
    np.testing.assert_array_equal(out, rout)
    assert lib.sdp_last_status() == 0, lib.sdp_last_error()


def test_calibration_oracle_chain_recovers_gains():
    """Pins the oracle for gain calibration: the reference's compiled normal
    equations, SUQ product and gain update (gains_calibration_run.c), with
    numpy's SVD in place of LAPACK's gesvd, recover known gains up to the
    free common phase within a few cycles."""
    ref = _ref()
    cfg = O.make_config(64, 1.0, 1.0, 8)
    rng = np.random.default_rng(3)
    nrx = 16
    pairs = np.array([(a, b) for a in range(nrx) for b in range(a + 1, nrx)] * 2, np.int32)
    nbl, n = pairs.shape[0], 2 * nrx
    g_true = (1.0 + 0.1 * rng.standard_normal(nrx)) * np.exp(1j * 0.3 * rng.standard_normal(nrx))
    pred = rng.standard_normal(nbl) + 1j * rng.standard_normal(nbl)
    meas = pred * g_true[pairs[:, 0]] * np.conj(g_true[pairs[:, 1]])
    c2 = lambda z: np.ascontiguousarray(np.stack([z.real, z.imag], 1).astype(np.float32))  # noqa: E731
    m2, p2 = c2(meas), c2(pred)
    g = c2(np.ones(nrx, complex))
    tok = _i(1)
    for _ in range(8):
        A = np.zeros((n, n), np.float32)
        Q = np.zeros(n, np.float32)
        ref.update_gain_calibration_actor(_i(nbl), _i(nrx), _i(nbl), C.byref(tok), m2.ctypes.data_as(_p),
                                          p2.ctypes.data_as(_p), g.ctypes.data_as(_p), pairs.ctypes.data_as(_p),
                                          C.byref(cfg), A.ctypes.data_as(_p), Q.ctypes.data_as(_p))
        assert np.array_equal(A, A.T)
        u, s, vt = np.linalg.svd(A.astype(np.float64).T)
        S = s.astype(np.float32)
        U = np.ascontiguousarray(u.T).astype(np.float32)    # LAPACK's column-major U
        VT = np.ascontiguousarray(vt.T).astype(np.float32)  # and V^T
        suq = np.zeros(n, np.float32)
        ref.calculate_SUQ_product_actor(_i(n), _i(n), S.ctypes.data_as(_p), U.ctypes.data_as(_p),
                                        Q.ctypes.data_as(_p), C.byref(cfg), suq.ctypes.data_as(_p))
        out = np.zeros((nrx, 2), np.float32)
        ref.calculate_delta_update_gains_actor(_i(n), _i(nrx), suq.ctypes.data_as(_p), VT.ctypes.data_as(_p),
                                               C.byref(cfg), g.ctypes.data_as(_p), out.ctypes.data_as(_p))
        g = out
    est = g[:, 0] + 1j * g[:, 1]
    est = est * np.exp(-1j * np.angle(np.vdot(g_true, est)))
    assert np.abs(est - g_true).max() <= 2e-3
