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
