"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (str(ROOT), str(ROOT / "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run on a B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


def golden_paths():
    return sorted(GOLDEN.glob("*.npz"))


def load_golden(path):
    from back40computing_b200.graphs import CsrGraph
    z = np.load(path)
    g = CsrGraph(z["row_offsets"].astype(np.int32), z["column_indices"].astype(np.int32), path.stem)
    return g, z["sources"], z["labels"], z["depths"]


@pytest.fixture(scope="session")
def cuda_device():
    """Fails (never skips) when a GPU test runs without a visible CUDA device."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected but no CUDA device is visible")
    torch.cuda.init()
    return torch.cuda.current_device()
