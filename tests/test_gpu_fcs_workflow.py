"""The workflow's full-counting-statistics stage on the GPU
(workflow.run_fcs, workflow.compute_fcs_k_moments) against negfpy's own
_run_fcs (workflows/ifc_bulk.py:1690-1935, tests/golden/fcs.npz): the
silicon study's material under every x/y mode, temperature sweep and eta
scheme, and the inputs of negfpy's TaN FCS study run (150 omegas, 144/256 k,
30 layers, n = 24).

Bounds: the k moments within 1e-10 max(|ref|, 1) per omega with equal eta
choices and k counts; C1, C2 and the plotted y, y_std within 1e-10 of each
value, NaN where negfpy's Bose weights overflow (at 2 K)."""

from __future__ import annotations

import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from negfpy_b200 import workflow as WF  # noqa: E402
from negfpy_b200.models import MaterialKspaceParams, interface_contacts, material_kspace_device  # noqa: E402
from tests.conftest import GOLDEN  # noqa: E402
from tests.golden.make_golden import FCS_CFGS, FCS_KEYS  # noqa: E402

TOL = 1e-10


@pytest.fixture(scope="module")
def fix():
    return np.load(GOLDEN / "fcs.npz")


def _params(fix, p: str) -> MaterialKspaceParams:
    def terms(key):
        if f"{p}_{key}_keys" not in fix.files:
            return None
        return {tuple(int(x) for x in k): b for k, b in zip(fix[f"{p}_{key}_keys"], fix[f"{p}_{key}_blocks"])}

    return MaterialKspaceParams(masses=fix[f"{p}_masses"], fc00_terms=terms("fc00"), fc01_terms=terms("fc01"),
                                fc10_terms=terms("fc10"), dof_per_atom=int(fix[f"{p}_dof"]),
                                onsite_pinning=float(fix[f"{p}_pinning"]))


def _kmesh(fix, p: str) -> dict:
    km = json.loads(str(fix[f"{p}_kmesh"]))
    for part in ("low", "high"):
        km[part]["kpoints"] = [tuple(k) for k in km[part]["kpoints"]]
    return km


def _run(fix, p: str, cfg: dict) -> dict:
    prm = _params(fix, p)
    ll, lr, vdl_l, vdl_r = interface_contacts(prm)
    dev = material_kspace_device(n_layers=int(fix[f"{p}_n_layers"]), params=prm)
    return WF.run_fcs(cfg, omegas=fix[f"{p}_omegas"], kmesh=_kmesh(fix, p), device=dev, lead_left=ll, lead_right=lr,
                      device_to_lead_left=vdl_l, device_to_lead_right=vdl_r, area_m2=float(fix[f"{p}_area"]))


def _check(res: dict, fix, prefix: str) -> None:
    for key in FCS_KEYS:
        got, ref = np.asarray(res[key]), fix[f"{prefix}_{key}"]
        assert got.shape == ref.shape, key
        assert np.array_equal(np.isnan(got), np.isnan(ref)), key
        ok = ~np.isnan(ref)
        if key in ("n_k_success", "eta_selected", "x", "temp_left_k", "temp_right_k"):
            assert np.array_equal(got[ok], ref[ok]), key
        elif key in ("t_mean", "t2_mean"):
            err = np.abs(got[ok] - ref[ok]) / np.maximum(np.abs(ref[ok]), 1.0)
            assert err.max(initial=0.0) <= TOL, (key, float(err.max()))
        else:
            err = np.abs(got[ok] - ref[ok]) / np.maximum(np.abs(ref[ok]), 1e-300)
            assert err.max(initial=0.0) <= TOL, (key, int(np.argmax(err)), float(err.max()))
    assert res["omega_failures"] == json.loads(str(fix[f"{prefix}_failures"]))


@pytest.mark.parametrize("name", list(FCS_CFGS))
def test_fcs_stage_variants(fix, name):
    _check(_run(fix, "si", FCS_CFGS[name]), fix, name)


def test_fcs_stage_on_the_tan_study(fix):
    cfg = json.loads(str(fix["tan_cfg"]))
    cfg["solver"]["surface_gf_method"] = "sancho_rubio"
    _check(_run(fix, "tan", cfg), fix, "tan_sr")

