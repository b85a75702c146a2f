"""Shared test set-up.

* registers the ``gpu`` marker (tests that need a CUDA device);
* puts the package directory and oracle/ on sys.path;
* builds the oracle restatement and libsdp_b200.so when they are missing
  (nvcc and gcc are present wherever the tests run).

The oracle is the checker only: tests compare the CUDA path with it.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "simsdp-generic-imaging-pipeline_b200"
ORACLE = ROOT / "oracle"
GOLDEN = Path(__file__).resolve().parent / "golden"
for p in (PKG, ORACLE):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the libsdp_b200 kernels)")


def _ensure_oracle():
    if not (ORACLE / "_build" / "liboracle_f32.so").exists() or not (ORACLE / "_build" / "liboracle_f64.so").exists():
        subprocess.run(["make", "-s", "-C", str(ORACLE), "all"], check=True)


def _ensure_lib():
    if not (PKG / "libsdp_b200.so").exists():
        subprocess.run([sys.executable, str(PKG / "build.py")], check=True)


@pytest.fixture(scope="session")
def oracle32():
    _ensure_oracle()
    import oracle
    return oracle.Oracle("f32")


@pytest.fixture(scope="session")
def oracle64():
    _ensure_oracle()
    import oracle
    return oracle.Oracle("f64")


@pytest.fixture(scope="session")
def sdp():
    _ensure_lib()
    import sdp_b200
    return sdp_b200


@pytest.fixture(scope="session")
def actors(sdp):
    import torch
    assert torch.cuda.is_available(), "gpu tests need a CUDA device"
    return sdp.Actors()


@pytest.fixture(scope="session")
def device(sdp):
    import torch
    assert torch.cuda.is_available(), "gpu tests need a CUDA device"
    torch.cuda.init()
    return sdp.Device()


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return dict(np.load(GOLDEN / name))
    return load


def rel_rms(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))
