"""The workflow's transmission stage (batched ladders on the GPU) against
negfpy's own _run_transmission on the same inputs (tests/golden/workflow.npz):
values, eta records, failure records, rejection counts and summary."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from negfpy_b200 import workflow as WF  # noqa: E402
from negfpy_b200.models import MaterialKspaceParams, material_kspace_device, material_kspace_lead  # noqa: E402

GOLDEN = Path(__file__).parent / "golden"


def _load_make_golden():
    import importlib.util

    spec = importlib.util.spec_from_file_location("make_golden", GOLDEN / "make_golden.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="module")
def setup():
    mg = _load_make_golden()
    dev, lead = mg.workflow_system(MaterialKspaceParams, material_kspace_lead, material_kspace_device)
    return mg, dev, lead, np.load(GOLDEN / "workflow.npz")


def _norm(obj):
    return json.loads(json.dumps(obj, default=lambda o: list(o) if isinstance(o, tuple) else o))


def _close(a, b, rel):
    if isinstance(a, dict):
        assert set(a) == set(b), (a, b)
        for k in a:
            _close(a[k], b[k], rel)
    elif isinstance(a, list):
        assert len(a) == len(b)
        for x, y in zip(a, b):
            _close(x, y, rel)
    elif isinstance(a, float) and isinstance(b, (float, int)):
        assert abs(a - b) <= rel * max(1.0, abs(b)), (a, b)
    else:
        assert a == b, (a, b)


@pytest.mark.parametrize("name", ["adaptive", "global", "fixed", "strict", "strict_global"])
def test_run_transmission_matches_negfpy(setup, name):
    mg, dev, lead, gold = setup
    res = WF.run_transmission(mg.WORKFLOW_CFGS[name], device=dev, lead_left=lead, lead_right=lead,
                              omegas=np.array(mg.WORKFLOW_OMEGAS), kmesh=mg.WORKFLOW_KMESH)
    ref_v = gold[name + "_values"]
    v = res["values"]
    assert np.array_equal(np.isnan(v), np.isnan(ref_v))
    ok = ~np.isnan(ref_v)
    scale = max(1.0, float(np.abs(ref_v[ok]).max())) if ok.any() else 1.0
    assert float(np.abs(v[ok] - ref_v[ok]).max(initial=0.0)) <= 1e-10 * scale
    meta = json.loads(str(gold[name + "_meta"]))
    ours = _norm({k: res[k] for k in ("eta_records", "omega_failures", "n_rejected_total", "summary")})
    ours["summary"]["parallel"]["workers"] = meta["summary"]["parallel"]["workers"]  # host core count differs
    _close(ours, meta, 1e-12)
