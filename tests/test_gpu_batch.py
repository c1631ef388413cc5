"""Uneven batch in one persistent launch: every item against the per-system
FP64 path and a sample against the oracle, the mixed precision against
FP64, CUDA-graph replay, out-of-range items, a system with different leads,
and the autotuner on the GPU."""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from negfpy_b200 import engine, workloads as W  # noqa: E402
from negfpy_b200.batch import Items, UnevenBatch  # noqa: E402

TOL_T = 1e-10


@pytest.fixture(scope="module")
def small():
    ws = W.uneven_workload(seed=7, n_systems=6, n_omega=12, k_range=(1, 5), layer_range=(3, 12),
                           orders=(24, 48, 72, 96))
    return ws, UnevenBatch(ws)


def _reference(ws):
    out = []
    for w in ws:
        s = engine.StackedSystem.from_arrays(w.lead_l, w.lead_l, w.onsite, w.coupling, w.n_layers, same_leads=True)
        K = len(w.kpoints)
        om = torch.as_tensor(np.repeat(w.omegas, K), device="cuda")
        ki = torch.as_tensor(np.tile(np.arange(K), w.omegas.size), device="cuda", dtype=torch.int32)
        r = s.transmission(om, ki, torch.full_like(om, w.eta))
        assert int((r["status"] != 0).sum()) == 0
        out.append(r["T"])
    return torch.cat(out)


def test_batch_f64_matches_per_system_path(small):
    ws, b = small
    ref = _reference(ws)
    for order in ("lpt", "interleave", "system"):
        it = b.items([w.omegas for w in ws], order)
        r = b.solve(it, "f64")
        assert int((r["status"] != 0).sum()) == 0
        err = float(((r["T"] - ref).abs() / ref.abs().clamp_min(1.0)).max())
        assert err <= TOL_T, (order, err)


def test_batch_matches_oracle_sample(small):
    from oracle.negf_oracle import transmission_point

    ws, b = small
    it = b.items([w.omegas for w in ws], "lpt")
    T = b.solve(it, "f64")["T"].cpu().numpy()
    offs = np.cumsum([0] + [w.omegas.size * len(w.kpoints) for w in ws])
    for si in (0, 3, 5):
        w = ws[si]
        K = len(w.kpoints)
        for wi, ki in ((2, 0), (9, K - 1)):
            ref = transmission_point(w.omegas[wi], [w.onsite[ki, 0]] * w.n_layers,
                                     [w.coupling[ki, 0]] * (w.n_layers - 1),
                                     (w.lead_l["d00"][ki], w.lead_l["d01"][ki], w.lead_l["d10"][ki]),
                                     (w.lead_l["d00"][ki], w.lead_l["d01"][ki], w.lead_l["d10"][ki]), eta=w.eta)
            got = T[offs[si] + wi * K + ki]
            assert abs(got - ref) <= TOL_T * max(1.0, abs(ref)), (si, wi, ki, got, ref)


def test_batch_mixed_against_f64(small):
    ws, b = small
    it = b.items([w.omegas for w in ws], "lpt")
    r64 = b.solve(it, "f64")
    rr = b.solve(it, "mixed_fallback")
    assert int((rr["status"] != 0).sum()) == 0
    err = float(((rr["T"] - r64["T"]).abs() / r64["T"].abs().clamp_min(1.0)).max())
    assert err <= 1e-3, err
    r2 = b.solve(it, "f64", blocks_per_sm=2)
    assert float(((r2["T"] - r64["T"]).abs() / r64["T"].abs().clamp_min(1.0)).max()) <= TOL_T


def test_batch_graph_replay(small):
    ws, b = small
    it = b.items([w.omegas for w in ws], "lpt")
    direct, _, _ = b.launch(it, "f64")
    direct = direct.clone()
    g, (T, st, iters) = b.graph(it, "f64")
    T.fill_(-1.0)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(T, direct) and int((st != 0).sum()) == 0
    T.fill_(-1.0)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(T, direct)


def test_batch_out_of_range_items(small):
    ws, b = small
    it = b.items([w.omegas[:2] for w in ws], "system")
    sysv, kv = it.system.clone(), it.k.clone()
    sysv[0] = b.n_systems            # no such system
    kv[1] = len(ws[int(sysv[1])].kpoints)  # k outside the system's grid
    bad = Items(sysv, kv, it.omega, it.perm, it.cost)
    T, st, _ = b.launch(bad, "f64")
    T0, st0, _ = b.launch(it, "f64")
    assert int(st[0]) == 5 and int(st[1]) == 5 and bool(torch.isnan(T[:2]).all())
    assert torch.equal(T[2:], T0[2:]) and int((st[2:] != 0).sum()) == 0


def test_batch_with_different_leads():
    from negfpy_b200 import adjoint
    from negfpy_b200.workloads import Workload

    pr = adjoint.hetero_problem(n_k=3, n_omega=10)
    m = pr.model
    theta = torch.as_tensor(m.theta0, device="cuda")
    on, cp = m.blocks(theta, pr.kpoints)
    la, lb = m.lead_blocks("A", pr.kpoints), m.lead_blocks("B", pr.kpoints)
    om = pr.om.cpu().numpy()
    eta = float(pr.eta[0])
    hw = Workload("hetero", om, pr.kpoints, {k: la[k] for k in ("d00", "d01", "d10")},
                  {k: lb[k] for k in ("d00", "d01", "d10")}, on.cpu().numpy(), cp.cpu().numpy(), m.L, eta=eta,
                  same_leads=False, vl=pr.vl.cpu().numpy(), vr=pr.vr.cpu().numpy())
    other = W.uneven_workload(seed=9, n_systems=2, n_omega=10, k_range=(1, 3), layer_range=(3, 6), orders=(24,))
    b = UnevenBatch([hw] + other)
    it = b.items([om] + [w.omegas for w in other], "lpt")
    r = b.solve(it, "f64")
    P = om.size * len(pr.kpoints)
    ref = pr.transmission_theta(theta).reshape(-1)
    err = float(((r["T"][:P] - ref).abs() / ref.abs().clamp_min(1.0)).max())
    assert err <= TOL_T, err


def test_tuner_on_gpu(small, tmp_path):
    from negfpy_b200.autotune import BatchTuner

    ws, b = small
    tuner = BatchTuner(tmp_path / "tune.json")
    c = tuner.tune(b, "mixed", [w.omegas[:3] for w in ws], reps=1)
    assert c["blocks_per_sm"] in (1, 2) and c["order"] in ("lpt", "interleave", "system") and not c["cached"]
    assert tuner.tune(b, "mixed", [w.omegas[:3] for w in ws])["cached"]


def test_split_schedule_matches_single_launch(small, tmp_path):
    """The split schedule (one launch per padded-order class, each with its
    own tuned launch shape and order) gives every item bitwise the same T as
    the single launch, directly and replayed from its CUDA graph; the tuner
    returns one cached entry per class."""
    from negfpy_b200.autotune import BatchTuner

    ws, b = small
    it = b.items([w.omegas for w in ws], "lpt")
    T1, s1, _ = b.launch(it, "f64")
    single = torch.empty_like(T1)
    single[it.perm] = T1
    tuner = BatchTuner(tmp_path / "tune.json")
    plan = tuner.tune_split(b, "f64", [w.omegas[:2] for w in ws], reps=1)
    assert sorted(plan) == sorted(set(int(c) for c in b.sys_class))
    assert all(e["blocks_per_sm"] in (1, 2) and not e["cached"] for e in plan.values())
    assert all(e["cached"] for e in tuner.tune_split(b, "f64", [w.omegas[:2] for w in ws]).values())
    parts = b.split_parts(it, plan)
    assert sum(int(sub.system.numel()) for _, _, sub, _ in parts) == int(it.system.numel())
    T2, s2, _ = b.launch_split(parts, "f64")
    assert torch.equal(T2, single) and int((s2 != 0).sum()) == 0
    g, (T3, _, _) = b.graph_split(parts, "f64")
    T3.fill_(-1.0)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(T3, single)
    b.release(g)
