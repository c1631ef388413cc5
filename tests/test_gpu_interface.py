"""The IFC transport set-up (negfpy ``workflows/ifc_bulk.py:690-742``) on the
GPU: blocks of the batched builder against the host builder, T through
``transmission_grid`` (GPU-built and host-built blocks) against negfpy's, and
the workflow's transmission stage with these contacts against negfpy's
``_run_transmission`` (``tests/golden/interface.npz``)."""

from __future__ import annotations

import json

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

import negfpy_b200 as nb  # noqa: E402
from negfpy_b200 import workflow as WF  # noqa: E402
from negfpy_b200.kspace import interface_system  # noqa: E402
from negfpy_b200.models import interface_contacts, material_kspace_device  # noqa: E402
from tests.conftest import GOLDEN, rel_err  # noqa: E402
from tests.golden.make_golden import (INTERFACE_LAYERS, WORKFLOW_CFGS, WORKFLOW_KMESH,  # noqa: E402
                                      WORKFLOW_OMEGAS)
from tests.test_gpu_workflow import _close, _norm  # noqa: E402
from tests.test_interface_host import NAMES, kpoints_of, params_of  # noqa: E402


@pytest.fixture(scope="module")
def fix():
    return np.load(GOLDEN / "interface.npz")


@pytest.mark.parametrize("name", NAMES)
def test_gpu_blocks_match_host_builder(fix, name):
    prm = params_of(fix, name)
    kp = kpoints_of(name)
    L = INTERFACE_LAYERS[name]
    s = interface_system(prm, {"n_layers": L, "layer_masses": None}, kp)
    ll, lr, vdl_l, vdl_r = interface_contacts(prm)
    dev = material_kspace_device(L, prm)

    def close(got: torch.Tensor, ref: np.ndarray):
        ref = np.asarray(ref)
        assert np.abs(got.cpu().numpy() - ref).max() <= 1e-14 * np.abs(ref).max()

    assert not s.same_leads
    for j, k in enumerate(kp):
        for lead, blocks in ((ll, s.lead_l), (lr, s.lead_r)):
            for i in range(3):
                close(blocks[i][j], lead.blocks(k)[i])
        close(s.vl[j], vdl_l(k))
        close(s.vr[j], vdl_r(k))
        d = dev.device(k)
        close(s.onsite[j, 0], d.onsite_blocks[0])
        close(s.coupling[j, 0], d.coupling_blocks[0])


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("route", ["gpu_blocks", "host_blocks"])
def test_transmission_grid_matches_negfpy(fix, name, route):
    """T[w, k] through the contacts, within 1e-10 max(|T|, 1) of negfpy.  An
    omega scale of 1 (exact) sends the grid through the per-k host builders."""
    prm = params_of(fix, name)
    L = INTERFACE_LAYERS[name]
    ll, lr, vdl_l, vdl_r = interface_contacts(prm)
    dev = material_kspace_device(L, prm)
    r = nb.transmission_grid(fix[f"{name}_omegas"], kpoints_of(name), dev, ll, lr, eta=float(fix[f"{name}_eta"]),
                             device_to_lead_left=vdl_l, device_to_lead_right=vdl_r,
                             omega_scale=None if route == "gpu_blocks" else 1.0)
    assert np.all(r["status"] == 0)
    assert rel_err(r["T"], fix[f"{name}_T"]).max() <= 1e-10


def test_workflow_with_interface_contacts_matches_negfpy(fix):
    prm = params_of(fix, "slab")
    ll, lr, vdl_l, vdl_r = WF._build_interface_contacts(prm)
    dev = material_kspace_device(4, prm)
    res = WF.run_transmission(WORKFLOW_CFGS["adaptive"], device=dev, lead_left=ll, lead_right=lr,
                              device_to_lead_left=vdl_l, device_to_lead_right=vdl_r,
                              omegas=np.array(WORKFLOW_OMEGAS), kmesh=WORKFLOW_KMESH)
    ref_v = fix["workflow_values"]
    v = res["values"]
    assert np.array_equal(np.isnan(v), np.isnan(ref_v))
    ok = ~np.isnan(ref_v)
    scale = max(1.0, float(np.abs(ref_v[ok]).max()))
    assert float(np.abs(v[ok] - ref_v[ok]).max(initial=0.0)) <= 1e-10 * scale
    meta = json.loads(str(fix["workflow_meta"]))
    ours = _norm({k: res[k] for k in ("eta_records", "omega_failures", "n_rejected_total", "summary")})
    ours["summary"]["parallel"]["workers"] = meta["summary"]["parallel"]["workers"]  # host core count differs
    _close(ours, meta, 1e-12)


def test_per_omega_ladders_match_negfpy(fix):
    """transmission_kavg and both eta ladders through the contacts (all k
    blocks built on the GPU once per call) against negfpy's values and info
    dictionaries, rejected records included."""
    prm = params_of(fix, "slab")
    ll, lr, vdl_l, vdl_r = interface_contacts(prm)
    dev = material_kspace_device(4, prm)
    kp = kpoints_of("slab")
    w = float(fix["slab_omegas"][1])
    kw = dict(device_to_lead_left=vdl_l, device_to_lead_right=vdl_r)
    ladder = tuple(float(x) for x in fix["ladder"])
    t = nb.transmission_kavg(w, dev, ll, lr, kpoints=kp, eta=float(fix["slab_eta"]), **kw)
    assert abs(t - float(fix["kavg"])) <= 1e-10 * max(1.0, abs(float(fix["kavg"])))
    for key, fn, extra in (("adaptive", nb.transmission_kavg_adaptive, {}),
                           ("global", nb.transmission_kavg_adaptive_global_eta, {"min_success_fraction": 0.3})):
        val, info = fn(w, dev, ll, lr, kpoints=kp, eta_values=ladder, max_channel_factor=0.2, collect_rejected=True,
                       **kw, **extra)
        ref = float(fix[key + "_value"])
        assert abs(val - ref) <= 1e-10 * max(1.0, abs(ref)), key
        _close(_norm(info), json.loads(str(fix[key + "_info"])), 1e-10)
