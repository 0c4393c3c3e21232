"""Shared test configuration.

Markers: ``gpu`` tests need a CUDA device and the built library; every other test runs on CPU.
Every test starts from seeded NumPy / torch generators.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built CUDA library")


@pytest.fixture(autouse=True)
def _seed_everything():
    np.random.seed(0)
    try:
        import torch
    except ModuleNotFoundError:
        pass
    else:
        torch.manual_seed(0)
    yield


def golden(name: str):
    return np.load(GOLDEN / name)


def golden_names(prefix: str):
    return sorted(p.name for p in GOLDEN.glob(f"{prefix}*.npz"))
