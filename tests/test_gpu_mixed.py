"""Mixed-precision device solve (FP32 sweep on 3 x TF32 tensor-core products,
FP64 self-energies, broadenings and trace) against the FP64 kernel.

The FP32 sweep is not held to the FP64 parity bound.  Its error against the
FP64 path (same surface GFs) is bounded here at the measured level with a
margin: |dT| <= tol * max(1, |T|) with tol 1e-5 for the chain, 1e-4 for the
n = 48 slab and 1e-3 for the n = 96 bulk and the 48 | 72 heterojunction, and
the relative error of kappa(300 K) on the sampled grids below 2e-5.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from negfpy_b200 import engine, workloads as W  # noqa: E402
from negfpy_b200.adjoint import kappa_weights  # noqa: E402


def _points(wl, wi):
    K = len(wl.kpoints)
    om = torch.as_tensor(np.repeat(wl.omegas[wi], K), device="cuda")
    ki = torch.as_tensor(np.tile(np.arange(K), len(wi)), device="cuda", dtype=torch.int32)
    return om, ki, torch.full_like(om, wl.eta)


def _both(wl, wi):
    s = engine.StackedSystem.from_arrays(wl.lead_l, wl.lead_l, wl.onsite, wl.coupling, wl.n_layers, same_leads=True)
    om, ki, eta = _points(wl, wi)
    rl = engine.sgf_sr(*s.lead_l, om, eta, ki)
    args = (s.onsite, s.coupling, s.n_layers, s.vl, s.vr, rl["g"], rl["g"], om, eta, ki, rl["status"])
    t64, s64 = engine.rgf_transmission(*args)
    tm, sm = engine.rgf_transmission(*args, precision="mixed")
    assert int((s64 != 0).sum()) == 0 and int((sm != 0).sum()) == 0
    return t64, tm, args


def _kappa(wl, wi, t):
    w = kappa_weights(torch.as_tensor(wl.omegas[wi], device="cuda"), 300.0, wl.omega_unit_rad_s)
    return float((w * t.reshape(len(wi), len(wl.kpoints)).mean(1)).sum())


@pytest.mark.parametrize("name,wl_fn,stride,tol", [
    ("chain", W.chain_workload, 7, 1e-5),
    ("slab48", W.slab_workload, 64, 1e-4),
    ("bulk96", W.bulk_workload, 256, 1e-3),
])
def test_mixed_matches_f64(name, wl_fn, stride, tol):
    wl = wl_fn()
    wi = np.arange(0, wl.omegas.size, stride)
    t64, tm, _ = _both(wl, wi)
    err = float(((tm - t64).abs() / t64.abs().clamp_min(1.0)).max())
    assert err <= tol, (name, err)
    k64, km = _kappa(wl, wi, t64), _kappa(wl, wi, tm)
    assert abs(km - k64) <= 2e-5 * abs(k64), (name, km, k64)


def test_mixed_heterojunction_layer_resolved():
    from negfpy_b200 import adjoint
    pr = adjoint.hetero_problem(n_k=4, n_omega=64)
    theta = torch.as_tensor(pr.model.theta0, device="cuda")
    on, cp = pr.model.blocks(theta, pr.kpoints)
    args = (on.contiguous(), cp.contiguous(), pr.model.L, pr.vl, pr.vr, pr.g_l, pr.g_r, pr.omega, pr.eta, pr.ki,
            pr.lead_status)
    t64, _ = engine.rgf_transmission(*args)
    tm, sm = engine.rgf_transmission(*args, precision="mixed")
    assert int((sm != 0).sum()) == 0
    err = float(((tm - t64).abs() / t64.abs().clamp_min(1.0)).max())
    assert err <= 1e-3, err


def test_mixed_fallback_and_lead_status():
    wl = W.slab_workload()
    wi = np.arange(5, wl.omegas.size, 256)
    t64, tm, args = _both(wl, wi)
    t, st, nb = engine.rgf_transmission_mixed(*args)
    assert nb == 0 and int((st != 0).sum()) == 0
    assert torch.equal(t, tm)
    # a failed lead skips the point and keeps its status; it is not re-solved
    lst = args[-1].clone()
    lst[3] = 1
    t2, st2, nb2 = engine.rgf_transmission_mixed(*args[:-1], lst)
    assert nb2 == 0 and int(st2[3]) == 1 and bool(torch.isnan(t2[3]))
    s = engine.StackedSystem.from_arrays(wl.lead_l, wl.lead_l, wl.onsite, wl.coupling, wl.n_layers, same_leads=True)
    om, ki, eta = _points(wl, wi)
    r = s.transmission(om, ki, eta, precision="mixed")
    assert r["fallback"] == 0 and torch.equal(r["T"], tm)


def test_precision_names():
    with pytest.raises(ValueError):
        engine.rgf_transmission(None, None, 1, None, None, None, None, torch.zeros(1), None, None, None,
                                precision="f16")
