"""Shared test setup: import paths, the `gpu` marker, common helpers."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "edegpredict-engine-rotary_b200"))
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and runs the CUDA path")


def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def max_rel(a, b, scale=None) -> float:
    """max |a - b| / scale, scale = max |b| unless given."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.size == 0:
        return 0.0
    s = float(np.abs(b).max()) if scale is None else float(scale)
    return float(np.abs(a - b).max() / max(s, 1e-300))


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle

    return Oracle()
