import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def golden_bulk():
    return dict(np.load(GOLDEN / "bulk.npz"))


@pytest.fixture(scope="session")
def golden():
    return {name: dict(np.load(GOLDEN / f"{name}.npz")) for name in ("chain", "slab", "cases")}


def rel_err(a, b, floor=1.0):
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    return np.abs(a - b) / np.maximum(np.abs(b), floor)
