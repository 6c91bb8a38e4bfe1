"""Shared test set-up: the `gpu` marker, native builds, common fixtures."""
from __future__ import annotations

import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


def _ensure_native():
    from sfr3d_b200 import build
    build.build_systems()
    if not os.path.exists(build.LIB) or os.environ.get("SFR_REBUILD"):
        build.build_cuda()
    oracle_dir = os.path.join(ROOT, "oracle")
    if not os.path.exists(os.path.join(oracle_dir, "liboracle.so")):
        subprocess.run(["make", "-s", "-C", oracle_dir], check=True)


_ensure_native()


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    if not gpu_available():
        pytest.fail("GPU test collected without a CUDA device")
    import torch
    torch.cuda.init()
    return torch


def rel(a, b):
    import numpy as np
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


@pytest.fixture(params=[1, 2], ids=["persistent", "graph"])
def engine(request):
    """Both solve engines: 1 = one cooperative launch, 2 = CUDA graph."""
    return request.param
