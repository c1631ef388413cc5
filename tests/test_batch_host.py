"""Host logic of the uneven batch (no GPU): the ctypes table layout against
the library's own sizeof, the item orders, the autotuner's selection and
cache, and the uneven workload generator."""

from __future__ import annotations

import ctypes as C
import json

import numpy as np
import pytest

from negfpy_b200 import _lib, workloads as W
from negfpy_b200.autotune import BatchTuner, batch_signature
from negfpy_b200.batch import NegfBatchSystem, item_cost, item_order


def test_table_record_matches_the_c_struct():
    lib = _lib.load()
    assert C.sizeof(NegfBatchSystem) == int(lib.negf_batch_system_bytes())
    assert NegfBatchSystem.onsite.offset == 24 and NegfBatchSystem.eta_device.offset == C.sizeof(NegfBatchSystem) - 8


def test_item_orders():
    system = np.array([0, 0, 0, 1, 1, 2])
    cost = np.array([1.0, 1.0, 1.0, 5.0, 5.0, 3.0])
    assert list(item_order(system, cost, "lpt")) == [3, 4, 5, 0, 1, 2]
    assert list(item_order(system, cost, "system")) == [0, 1, 2, 3, 4, 5]
    assert list(item_order(system, cost, "interleave")) == [0, 3, 5, 1, 4, 2]
    with pytest.raises(ValueError):
        item_order(system, cost, "random")
    assert item_cost(96, 96, 96, 40, True) > item_cost(48, 48, 48, 40, True) > 0
    assert item_cost(72, 48, 72, 30, False) > item_cost(72, 48, 72, 30, True)


def test_tuner_selects_the_fastest_and_caches(tmp_path):
    path = tmp_path / "tune.json"
    tuner = BatchTuner(path)
    times = {(1, "lpt"): 5.0, (1, "interleave"): 6.0, (1, "system"): 9.0, (2, "lpt"): 4.0,
             (2, "interleave"): float("inf"), (2, "system"): 7.0}
    calls = []

    def measure(bps, order):
        calls.append((bps, order))
        if np.isinf(times[(bps, order)]):
            raise RuntimeError("shape not available")
        return times[(bps, order)]

    key = batch_signature([(48, 48, 48, 20, 64, 1)], "f64", "gpu")
    r = tuner.select(key, measure)
    assert (r["blocks_per_sm"], r["order"], r["cached"]) == (2, "lpt", False)
    assert len(calls) == 6
    assert json.loads(path.read_text())[key]["order"] == "lpt"
    r2 = BatchTuner(path).select(key, measure)
    assert r2["cached"] and len(calls) == 6
    r3 = tuner.select(key, measure, force=True)
    assert not r3["cached"] and len(calls) == 12
    assert batch_signature([(1, 1, 1, 2, 3, 1), (4, 4, 4, 5, 6, 1)], "f64", "g") == \
        batch_signature([(4, 4, 4, 5, 6, 1), (1, 1, 1, 2, 3, 1)], "f64", "g")
    with pytest.raises(RuntimeError):
        BatchTuner(tmp_path / "x.json").select("k", lambda b, o: float("inf"))


def test_uneven_workload_shapes():
    ws = W.uneven_workload(seed=3, n_systems=6, n_omega=16, k_range=(1, 9), layer_range=(10, 60))
    assert len(ws) == 6
    for w in ws:
        assert w.n in W.UNEVEN_SHAPES and 10 <= w.n_layers <= 60 and 1 <= len(w.kpoints) <= 9
        assert w.omegas.size == 16 and w.omegas.max() <= 1.05 * w.omega_max + 1e-12
        d = w.lead_l["d00"][0]
        assert np.abs(d - d.conj().T).max() < 1e-12


def test_order_classes_and_split_parts():
    """Items grouped by padded block order, each class in its own item order,
    with the launch shape of its plan entry (a batch object without device
    state: class_items and split_parts are host logic)."""
    import torch

    from negfpy_b200.batch import Items, UnevenBatch, order_class

    assert [order_class(24, 24, 24), order_class(48, 48, 48), order_class(72, 48, 72), order_class(120, 96, 96)] == \
        [32, 48, 80, 128]
    b = UnevenBatch.__new__(UnevenBatch)
    b.device = torch.device("cpu")
    b.sys_class = np.array([32, 48, 32, 192])
    b.sys_order = np.array([24, 48, 30, 192])
    system = np.array([0, 1, 2, 3, 0, 3, 2])
    cost = np.array([1.0, 2.0, 3.0, 9.0, 1.5, 8.0, 0.5])
    it = Items(torch.as_tensor(system, dtype=torch.int32), torch.zeros(7, dtype=torch.int32),
               torch.arange(7, dtype=torch.float64), torch.arange(7) + 100, cost)
    parts = b.split_parts(it, {192: {"blocks_per_sm": 2, "order": "system"}})
    assert [(c, mo, bps) for c, mo, _, bps in parts] == [(32, 30, 1), (48, 48, 1), (192, 192, 2)]
    sub32 = parts[0][2]
    assert list(sub32.perm.numpy()) == [102, 104, 100, 106]  # lpt inside the class: costs 3, 1.5, 1, 0.5
    assert list(parts[2][2].perm.numpy()) == [103, 105]        # "system": the given order
    assert sum(int(p[2].system.numel()) for p in parts) == 7


def test_sum_by_k_groups_points_in_order():
    """The per-k reduction of per-point adjoint blocks (host side of the
    reproducible gradients): each k gets the sum of exactly its points, all
    into slot 0 when there is one slot or no k index, and a repeat gives the
    same bits."""
    import torch

    from negfpy_b200.engine import _sum_by_k

    gen = torch.Generator().manual_seed(5)
    src = torch.randn((9, 2, 3), dtype=torch.complex128, generator=gen)
    kidx = torch.tensor([2, 0, 2, 1, 0, 2, 1, 1, 0], dtype=torch.int32)
    dst = torch.zeros((3, 2, 3), dtype=torch.complex128)
    _sum_by_k(dst, src, kidx)
    for k in range(3):
        assert torch.allclose(dst[k], src[kidx == k].sum(0), rtol=0, atol=1e-14)
    again = torch.zeros_like(dst)
    _sum_by_k(again, src, kidx)
    assert torch.equal(again, dst)
    one = torch.zeros((1, 2, 3), dtype=torch.complex128)
    _sum_by_k(one, src, kidx)
    assert torch.allclose(one[0], src.sum(0), rtol=0, atol=1e-14)
    none = torch.zeros((1, 2, 3), dtype=torch.complex128)
    _sum_by_k(none, src, None)
    assert torch.equal(none, one)
