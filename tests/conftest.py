"""Shared fixtures: the CPU oracle, the golden vectors and the native library."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def golden():
    d = ROOT / "tests" / "golden"
    manifest = json.loads((d / "golden.json").read_text())
    arrays = dict(np.load(d / "golden.npz"))
    return manifest, arrays


@pytest.fixture(scope="session")
def native():
    """The in-tree CUDA library; built here if missing (nvcc is on every box)."""
    from fhetoothpaste_b200 import _native, build
    build.build_gpu()
    return _native.lib()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected on a machine without CUDA")
    torch.cuda.init()
    return torch
