"""Shared pytest configuration.

Tests marked ``gpu`` need a CUDA device and the built ``libtopo_b200.so``;
everything else runs on the CPU (the oracle, host logic, library loading).
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built CUDA library")


def load_golden(name: str):
    return np.load(GOLDEN / f"{name}.npz", allow_pickle=False)


def csr_from(d, prefix):
    import scipy.sparse as sp

    return sp.csr_matrix((d[f"{prefix}_data"], d[f"{prefix}_indices"], d[f"{prefix}_indptr"]),
                         shape=tuple(d[f"{prefix}_shape"]))


@pytest.fixture(scope="session")
def golden():
    return load_golden


@pytest.fixture(scope="session")
def cuda_dev():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("CUDA device not available")
    return torch.device("cuda:0")
