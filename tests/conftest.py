"""Shared pytest setup.

Markers: `gpu` tests need a CUDA device (B200, sm_100a) and call the CUDA path
through its C ABI; everything else runs on the CPU.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))
sys.path.insert(0, str(ROOT / "oracle"))  # mlp_ref: the surrogate network's FP64 oracle


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device; exercises libes_cuda.so")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def gpu_available() -> bool:
    try:
        import torch
        return bool(torch.cuda.is_available())
    except Exception:
        return False


@pytest.fixture(scope="session")
def golden():
    def load(name: str):
        p = GOLDEN / name
        if p.suffix == ".npy":
            return np.load(p)
        return json.loads(p.read_text())
    return load


@pytest.fixture(scope="session")
def cuda_device():
    """Every GPU test goes through here: no device means a hard failure when the
    test was explicitly selected with -m gpu on a GPU machine, a skip otherwise."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    from elasticscattering_b200 import _native
    _native.cuda_lib()
    return 0
