"""Shared fixtures. GPU tests are marked ``gpu``; CPU tests cover the oracle and host logic."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device and the built library")


@pytest.fixture(scope="session")
def golden_grids() -> dict[str, np.ndarray]:
    with np.load(GOLDEN / "grids.npz") as z:
        return {k: np.asfortranarray(z[k]) for k in z.files}


@pytest.fixture(scope="session")
def reference_8x9() -> dict[str, np.ndarray]:
    with np.load(GOLDEN / "reference_8x9.npz") as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def oracle():
    from oracle.shim import SpatialDiscretizationModule

    return SpatialDiscretizationModule()


@pytest.fixture(scope="session")
def cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyeulerale_b200 import _lib

    _lib.load()  # fails loudly if the library is not built
    return torch
