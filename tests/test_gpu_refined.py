"""Refined device solve: FP32 block LU factors with FP64 iterative refinement
(negf_rgf_transmission_refined), against the FP64 kernel and the oracle.

The refinement is held to the FP64 parity bound: |dT| <= 1e-10 max(1, |T|)
against the FP64 kernel on the same surface GFs (chain, n = 48 slab, n = 96
bulk, the layer-resolved 48 | 72 heterojunction), kappa(300 K) of the sampled
grids within 1e-10, and the slab sample against negfpy's own T (golden
fixture).  A point that cannot converge reports NEGF_REFINE_FAIL and is
solved again in FP64.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from negfpy_b200 import _lib, engine, workloads as W  # noqa: E402
from negfpy_b200.adjoint import kappa_weights  # noqa: E402

TOL = 1e-10
GOLDEN = Path(__file__).resolve().parent / "golden"


def _points(wl, wi):
    K = len(wl.kpoints)
    om = torch.as_tensor(np.repeat(wl.omegas[wi], K), device="cuda")
    ki = torch.as_tensor(np.tile(np.arange(K), len(wi)), device="cuda", dtype=torch.int32)
    return om, ki, torch.full_like(om, wl.eta)


def _args(wl, wi):
    s = engine.StackedSystem.from_arrays(wl.lead_l, wl.lead_l, wl.onsite, wl.coupling, wl.n_layers, same_leads=True)
    om, ki, eta = _points(wl, wi)
    rl = engine.sgf_sr(*s.lead_l, om, eta, ki)
    return (s.onsite, s.coupling, s.n_layers, s.vl, s.vr, rl["g"], rl["g"], om, eta, ki, rl["status"])


def _kappa(wl, wi, t):
    w = kappa_weights(torch.as_tensor(wl.omegas[wi], device="cuda"), 300.0, wl.omega_unit_rad_s)
    return float((w * t.reshape(len(wi), len(wl.kpoints)).mean(1)).sum())


@pytest.mark.parametrize("name,wl_fn,stride", [
    ("chain", W.chain_workload, 7),
    ("slab48", W.slab_workload, 64),
    ("bulk96", W.bulk_workload, 256),
])
def test_refined_matches_f64(name, wl_fn, stride):
    wl = wl_fn()
    wi = np.arange(0, wl.omegas.size, stride)
    args = _args(wl, wi)
    t64, s64 = engine.rgf_transmission(*args)
    tr, sr, steps = engine.rgf_transmission_refine64(*args)
    assert int((s64 != 0).sum()) == 0 and int((sr != 0).sum()) == 0, (name, sr.unique())
    err = float(((tr - t64).abs() / t64.abs().clamp_min(1.0)).max())
    assert err <= TOL, (name, err)
    k64, kr = _kappa(wl, wi, t64), _kappa(wl, wi, tr)
    assert abs(kr - k64) <= 1e-10 * abs(k64), (name, kr, k64)
    st = steps.cpu().numpy()
    assert st.min() >= 1 and st.max() <= engine.REFINE_MAX_STEPS


def test_refined_heterojunction_layer_resolved():
    from negfpy_b200 import adjoint

    pr = adjoint.hetero_problem(n_k=4, n_omega=64)
    theta = torch.as_tensor(pr.model.theta0, device="cuda")
    on, cp = pr.model.blocks(theta, pr.kpoints)
    args = (on.contiguous(), cp.contiguous(), pr.model.L, pr.vl, pr.vr, pr.g_l, pr.g_r, pr.omega, pr.eta, pr.ki,
            pr.lead_status)
    t64, _ = engine.rgf_transmission(*args)
    tr, sr, _ = engine.rgf_transmission_refine64(*args)
    assert int((sr != 0).sum()) == 0
    err = float(((tr - t64).abs() / t64.abs().clamp_min(1.0)).max())
    assert err <= TOL, err


def test_refined_slab_against_negfpy_fixture():
    """negfpy's own T at 36 slab points (tests/golden/slab.npz)."""
    d = np.load(GOLDEN / "slab.npz", allow_pickle=False)
    lead = {"d00": d["d00"], "d01": d["d01"], "d10": d["d10"]}
    s = engine.StackedSystem.from_arrays(lead, lead, d["onsite"][:, None], d["coupling"][:, None], int(d["n_layers"]),
                                         same_leads=True)
    pairs = d["pairs"]
    wpos = {int(w): i for i, w in enumerate(d["wsel"])}
    kpos = {int(k): j for j, k in enumerate(d["ksel"])}
    om = torch.as_tensor([float(d["omegas"][wpos[int(w)]]) for w, _ in pairs], device="cuda", dtype=torch.float64)
    ki = torch.as_tensor([kpos[int(k)] for _, k in pairs], device="cuda", dtype=torch.int32)
    r = s.transmission(om, ki, torch.full_like(om, float(d["eta"])), precision="refined")
    assert r["fallback"] == 0
    t = r["T"].cpu().numpy()
    err = np.abs(t - d["T"]) / np.maximum(np.abs(d["T"]), 1.0)
    assert err.max() <= TOL, err.max()


def test_refine_fail_falls_back_to_f64():
    """A tolerance that no refinement step can meet makes every point report
    NEGF_REFINE_FAIL; rgf_transmission_refined then re-solves all of them in
    FP64 and returns the FP64 kernel's T."""
    wl = W.slab_workload()
    wi = np.arange(3, wl.omegas.size, 512)
    args = _args(wl, wi)
    t64, _ = engine.rgf_transmission(*args)
    _, st, steps = engine.rgf_transmission_refine64(*args, tol=1e-300, max_steps=1)
    assert bool((st == _lib.REFINE_FAIL).all()) and bool((steps == 1).all())
    t, st2, nb, _ = engine.rgf_transmission_refined(*args, tol=1e-300, max_steps=1)
    assert nb == t.numel() and int((st2 != 0).sum()) == 0
    assert torch.equal(t, t64)
    # a failed lead keeps its status and is not re-solved
    lst = args[-1].clone()
    lst[1] = _lib.MAXITER
    t3, st3, nb3, _ = engine.rgf_transmission_refined(*args[:-1], lst)
    assert nb3 == 0 and int(st3[1]) == _lib.MAXITER and bool(torch.isnan(t3[1]))


def test_stacked_system_precisions():
    wl = W.slab_workload()
    wi = np.arange(11, wl.omegas.size, 256)
    s = engine.StackedSystem.from_arrays(wl.lead_l, wl.lead_l, wl.onsite, wl.coupling, wl.n_layers, same_leads=True)
    om, ki, eta = _points(wl, wi)
    r64 = s.transmission(om, ki, eta)
    rr = s.transmission(om, ki, eta, precision="refined")
    assert rr["fallback"] == 0 and int(rr["steps"].min()) >= 1
    err = float(((rr["T"] - r64["T"]).abs() / r64["T"].abs().clamp_min(1.0)).max())
    assert err <= TOL, err


def test_transmission_grid_precisions():
    """The public grid call takes the precision: "refined" equals FP64 within
    the parity bound; "mixed" within the FP32 sweep's error."""
    import negfpy_b200 as nb
    from negfpy_b200.models import material_kspace_device, material_kspace_lead

    wl = W.slab_workload(n_omega=64, n_k=8, n_layers=6)
    params = W.spring_network(wl.meta["seed"], ny=wl.meta["ny"], nz=wl.meta["nz"], periodic_y=True)
    lead = material_kspace_lead(params)
    dev = material_kspace_device(6, params)
    om = wl.omegas[3::8]
    r64 = nb.transmission_grid(om, wl.kpoints, dev, lead, lead, eta=wl.eta)
    rr = nb.transmission_grid(om, wl.kpoints, dev, lead, lead, eta=wl.eta, precision="refined")
    rm = nb.transmission_grid(om, wl.kpoints, dev, lead, lead, eta=wl.eta, precision="mixed")
    assert rr["fallback"] == 0 and rr["steps"].min() >= 1
    scale = np.maximum(np.abs(r64["T"]), 1.0)
    assert (np.abs(rr["T"] - r64["T"]) / scale).max() <= TOL
    assert (np.abs(rm["T"] - r64["T"]) / scale).max() <= 1e-4
