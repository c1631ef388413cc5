"""Host parts of the workflow stage (no GPU): QE unit conversion, eta ladder
caps and configuration parsing, against negfpy's recorded results."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from negfpy_b200 import workflow as WF


@pytest.fixture(scope="module")
def golden():
    return np.load(Path(__file__).parent / "golden" / "workflow.npz")


def test_qe_units_match_recorded_wavenumbers(golden):
    recs = json.loads(str(golden["adaptive_meta"]))["eta_records"]
    for r in recs:
        assert float(WF.qe_omega_to_cm1(r["omega_qe"])) == pytest.approx(r["omega_cm1"], rel=1e-15)


def test_eta_cap():
    base = (1e-7, 1e-5, 1e-3)
    assert WF.resolve_eta_values_for_omega(1.0, 1e5, eta_values=base, max_eta_over_omega=None,
                                           eta_ratio_cm1_min=None) == base
    assert WF.resolve_eta_values_for_omega(0.5, 1e5, eta_values=base, max_eta_over_omega=1e-4,
                                           eta_ratio_cm1_min=None) == (1e-7, 1e-5)
    assert WF.resolve_eta_values_for_omega(0.5, 10.0, eta_values=base, max_eta_over_omega=1e-4,
                                           eta_ratio_cm1_min=50.0) == base
    assert WF.resolve_eta_values_for_omega(1e-3, 1e5, eta_values=base, max_eta_over_omega=1e-6,
                                           eta_ratio_cm1_min=None) == (1e-7,)


def test_parallel_config_and_errors():
    assert WF.resolve_parallel_solver_config({"parallel": {"enabled": True, "workers": 4}}) == \
        {"enabled": True, "backend": "thread", "workers": 4, "blas_threads": 1}
    with pytest.raises(ValueError, match="solver.parallel.backend"):
        WF.resolve_parallel_solver_config({"parallel": {"backend": "mpi"}})
    with pytest.raises(ValueError, match="omega_scale_mode"):
        WF.run_transmission({"solver": {"omega_scale_mode": "thz", "surface_gf_method": "sr"}}, device=None,
                            lead_left=None, lead_right=None, omegas=np.ones(1), kmesh={})
    with pytest.raises(NotImplementedError):
        WF.run_transmission({"solver": {}}, device=None, lead_left=None, lead_right=None, omegas=np.ones(1),
                            kmesh={})
