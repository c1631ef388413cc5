"""The oracle's full device Green's function against negfpy's
(tests/golden/green.npz, written by negfpy's device_green_function)."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from negfpy_b200 import workloads as W
from oracle.negf_oracle import device_green_point


@pytest.fixture(scope="module")
def green():
    return np.load(Path(__file__).parent / "golden" / "green.npz")


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_oracle_green_chain_and_rect(green):
    on = [np.array([[2.0 + 0j]])] * 6
    cp = [np.array([[-1.0 + 0j]])] * 5
    lead = (np.array([[2.0 + 0j]]), np.array([[-1.0 + 0j]]), None)
    g, sl, sr = device_green_point(1.1, on, cp, lead, lead, eta=1e-8)
    assert _rel(g, green["chain_G"]) < 1e-12 and _rel(sl, green["chain_SL"]) < 1e-12
    on = [np.diag([2.0, 100.0]).astype(complex)] * 4
    cp = [np.diag([-1.0, 0.0]).astype(complex)] * 3
    g, sl, sr = device_green_point(1.0, on, cp, lead, lead, eta=1e-8, vl=np.array([[-1.0]]), vr=np.array([[-1.0]]),
                                   idx_l=[0], idx_r=[6])
    assert _rel(g, green["rect_G"]) < 1e-12 and _rel(sr, green["rect_SR"]) < 1e-12
