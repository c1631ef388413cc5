"""The workflow's surface-DOS stage on the GPU (workflow.run_dos) against
negfpy's own _run_dos (workflows/ifc_bulk.py:908-948, 1290-1441;
tests/golden/dos_workflow.npz): the fixed, global and per-k eta schemes on
the right interface lead of the silicon study's material, with a negative
omega, the omega = 0 point where the decimation fails, and a lead with one
NaN k point (failure messages, success fractions and thresholds).

Bound: 1e-9 max(|DOS|, 1) per omega, as for the single-point DOS; equal eta
records, failure records and summary."""

from __future__ import annotations

import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from negfpy_b200 import workflow as WF  # noqa: E402
from negfpy_b200.models import interface_contacts  # noqa: E402
from negfpy_b200.types import LeadKSpace  # noqa: E402
from tests.conftest import GOLDEN  # noqa: E402
from tests.golden.make_golden import DOS_NAN_K, DOS_WORKFLOW_CFGS, SR_FAILURE_ORDERS, nan_at, sr_failure_blocks  # noqa: E402,E501
from tests.test_gpu_studies import study_params  # noqa: E402
from tests.test_gpu_workflow import _close, _norm  # noqa: E402

TOL = 1e-9


@pytest.fixture(scope="module")
def setup():
    fix = np.load(GOLDEN / "dos_workflow.npz")
    prm = study_params(np.load(GOLDEN / "studies.npz"), "silicon_x")
    km = json.loads(str(fix["kmesh"]))
    for part in ("low", "high"):
        km[part]["kpoints"] = [tuple(k) for k in km[part]["kpoints"]]
    _, lead, _, _ = interface_contacts(prm)
    bad = LeadKSpace(blocks_builder=nan_at(lead, km["high"]["kpoints"][DOS_NAN_K]))
    return fix, km, lead, bad


@pytest.mark.parametrize("name", list(DOS_WORKFLOW_CFGS))
def test_dos_stage_matches_negfpy(setup, name):
    fix, km, lead, bad = setup
    res = WF.run_dos(DOS_WORKFLOW_CFGS[name], lead=bad if name.startswith("nan") else lead, omegas=fix["omegas"],
                     kmesh=km)
    v, ref = np.asarray(res["values"]), fix[f"{name}_values"]
    assert np.array_equal(np.isnan(v), np.isnan(ref))
    ok = ~np.isnan(ref)
    err = np.abs(v[ok] - ref[ok]) / np.maximum(np.abs(ref[ok]), 1.0)
    assert err.max(initial=0.0) <= TOL, (name, float(err.max(initial=0.0)))
    _close(_norm({k: res[k] for k in ("eta_records", "omega_failures", "summary")}),
           json.loads(str(fix[f"{name}_meta"])), 1e-12)


@pytest.mark.parametrize("n", SR_FAILURE_ORDERS)
def test_decimation_failure_messages_match_negfpy(setup, n):
    """Overflow from finite blocks is negfpy's "numerically unstable", NaN
    blocks its "non-finite values", for the 1 x 1, shared-memory and
    global-workspace kernels (status NEGF_UNSTABLE / NEGF_NONFINITE)."""
    import negfpy_b200 as nb

    ref = json.loads(str(setup[0]["sr_failure_messages"]))
    for case, (d00, d01) in sr_failure_blocks(n).items():
        with pytest.raises(Exception) as info:
            nb.surface_gf(0.5, d00, d01, eta=1e-8, method="sancho_rubio")
        assert f"{type(info.value).__name__}: {info.value}" == ref[f"{case}_{n}"]
