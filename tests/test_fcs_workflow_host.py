"""Argument checks of the workflow's FCS stage (negfpy
workflows/ifc_bulk.py:1800-1813), which run on the host before any launch."""

from __future__ import annotations

import numpy as np
import pytest

from tests.conftest import GOLDEN
from tests.golden.make_golden import FCS_CFGS
from tests.test_gpu_fcs_workflow import _run


@pytest.fixture(scope="module")
def fix():
    return np.load(GOLDEN / "fcs.npz")


@pytest.mark.parametrize("bad,msg", [({"x": "omega"}, "fcs.x must be"), ({"y": "flux"}, "fcs.y must be one of"),
                                     ({"n_points": 1}, "fcs.n_points must be >= 2"),
                                     ({"measurement_time_s": 0.0}, "fcs.measurement_time_s must be positive")])
def test_fcs_stage_checks(fix, bad, msg):
    cfg = FCS_CFGS["delta_conductance"]
    with pytest.raises(ValueError, match=msg):
        _run(fix, "si", {**cfg, "fcs": {**cfg["fcs"], **bad}})


def test_stages_without_launches():
    """Paths of the DOS and FCS stages that negfpy settles before any solve
    (workflows/ifc_bulk.py:1290-1441, 1690-1784): a QEP surface-GF name is
    refused, negative omegas are NaN without a failure record (all of them:
    "DOS calculation failed for all omega points."), and omega <= 0 has zero
    k moments."""
    from negfpy_b200 import workflow as WF

    km = {"low_cm1": 100.0, "low": {"kpoints": [(0.0,)]}, "high": {"kpoints": [(0.0,)]}}
    with pytest.raises(NotImplementedError):
        WF.run_dos({"solver": {"surface_gf_method": "generalized_eigen_svd"}}, lead=None, omegas=[-1.0], kmesh=km)
    with pytest.raises(NotImplementedError):
        WF.compute_fcs_k_moments({"solver": {}}, device=None, lead_left=None, lead_right=None, omegas=[0.0],
                                 kmesh=km)
    with pytest.raises(RuntimeError, match="DOS calculation failed for all omega points"):
        WF.run_dos({"solver": {"surface_gf_method": "sr"}}, lead=None, omegas=[-1.0, -0.5], kmesh=km)
    res = WF.compute_fcs_k_moments({"solver": {"surface_gf_method": "sancho_rubio"}}, device=None, lead_left=None,
                                   lead_right=None, omegas=[-0.2, 0.0], kmesh=km)
    assert res["t_mean"].tolist() == [0.0, 0.0] and res["t2_mean"].tolist() == [0.0, 0.0]
    assert res["n_k_success"].tolist() == [0, 0] and res["omega_failures"] == []
    assert np.isnan(res["eta_selected"]).all()
