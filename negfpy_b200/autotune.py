"""Autotuner for the uneven-batch launch.

The batch kernel has two compiled launch shapes: registers uncapped (one
resident block per SM) or capped at 128 a thread (two resident blocks per SM:
one point's latency-bound pivot steps overlap another's products, at the
price of some spilling).  The item order decides how evenly the persistent
blocks finish: "lpt" (largest estimated cost first), "interleave"
(round-robin over systems) or "system" (system by system).  The tuner times
every (blocks_per_sm, order) pair on a small omega sample of the batch with
CUDA events, keeps the fastest, and caches the choice in a JSON file keyed by
the GPU, the precision and the shape of the batch (block orders, layer counts
and k counts of its systems).

``BatchTuner.tune_split`` makes the same choice per padded-order class for
the split schedule (one launch per class), so the launch shape and item
order can differ between block orders.

The FP32 device sweeps (mixed and refined precision) have two product
tilings for block orders up to 128: 16 x 16 warp tiles on mma.sync, or
128 x n tiles on the tcgen05 tensor cores with TMEM accumulators.
``ProductPathTuner`` times both on a sample of a system's points and sets
the faster one for that order (``negf_set_fp32_product_path``), cached the
same way.

Cache file: ``$NEGF_B200_TUNE_CACHE``, else ``~/.cache/negfpy_b200/autotune.json``.
"""

from __future__ import annotations

import hashlib
import json
import os
from pathlib import Path
from typing import Callable

import numpy as np

CANDIDATES = [(bps, order) for bps in (1, 2) for order in ("lpt", "interleave", "system")]


def default_cache_path() -> Path:
    env = os.environ.get("NEGF_B200_TUNE_CACHE")
    return Path(env) if env else Path.home() / ".cache" / "negfpy_b200" / "autotune.json"


def batch_signature(shapes, precision: str, gpu: str) -> str:
    """Stable key of a batch: GPU name, precision and the sorted (n, nl, nr, L, K, same_leads) shapes."""
    body = json.dumps({"gpu": gpu, "precision": precision, "shapes": sorted(list(map(list, shapes)))})
    return hashlib.sha1(body.encode()).hexdigest()


def batch_shapes(batch) -> list[tuple]:
    return [(s.n, s.nl, s.nr, s.n_layers, s.K, int(s.same_leads)) for s, _, _ in batch.systems]


class BatchTuner:
    def __init__(self, cache_path: str | Path | None = None, candidates=None):
        self.path = Path(cache_path) if cache_path is not None else default_cache_path()
        self.candidates = list(candidates or CANDIDATES)

    def _load(self) -> dict:
        try:
            return json.loads(self.path.read_text())
        except (OSError, ValueError):
            return {}

    def _store(self, key: str, entry: dict) -> None:
        data = self._load()
        data[key] = entry
        try:
            self.path.parent.mkdir(parents=True, exist_ok=True)
            tmp = self.path.with_suffix(".tmp")
            tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
            tmp.replace(self.path)
        except OSError:
            pass  # a read-only home: the choice is used, just not remembered

    def select(self, key: str, measure: Callable[[int, str], float], force: bool = False) -> dict:
        """The cached choice for ``key``, or the fastest candidate by ``measure(bps, order) -> ms``."""
        if not force:
            hit = self._load().get(key)
            if hit is not None and (hit["blocks_per_sm"], hit["order"]) in self.candidates:
                return dict(hit, cached=True)
        times = {}
        for bps, order in self.candidates:
            try:
                times[(bps, order)] = float(measure(bps, order))
            except RuntimeError:
                times[(bps, order)] = float("inf")  # a launch shape the GPU cannot run
        (bps, order), ms = min(times.items(), key=lambda kv: kv[1])
        if not np.isfinite(ms):
            raise RuntimeError("no batch launch shape could be run")
        entry = {"blocks_per_sm": bps, "order": order, "ms": ms,
                 "timings": {f"{b}/{o}": t for (b, o), t in times.items()}}
        self._store(key, entry)
        return dict(entry, cached=False)

    def tune(self, batch, precision: str, sample_omegas, reps: int = 2, force: bool = False) -> dict:
        """Choose (blocks_per_sm, order) for ``batch`` at ``precision`` ("f64" or
        "mixed") by timing one launch over the items of ``sample_omegas``."""
        import torch

        gpu = torch.cuda.get_device_name() + f"/{torch.cuda.get_device_properties(0).multi_processor_count}SM"
        key = batch_signature(batch_shapes(batch), precision, gpu)

        def measure(bps: int, order: str) -> float:
            if batch.max_grid(precision, bps) <= 0:
                raise RuntimeError("launch shape not available")
            it = batch.items(sample_omegas, order)
            batch.launch(it, precision, blocks_per_sm=bps)  # warm-up
            best = float("inf")
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                batch.launch(it, precision, blocks_per_sm=bps)
                e1.record()
                torch.cuda.synchronize()
                best = min(best, e0.elapsed_time(e1))
            return best

        return self.select(key, measure, force)

    def tune_split(self, batch, precision: str, sample_omegas, reps: int = 2, force: bool = False) -> dict:
        """The split schedule's plan: for every order class of ``batch`` the
        (blocks_per_sm, order) that runs the class's items of
        ``sample_omegas`` fastest on their own (launched with the class's
        largest order), each cached under the shapes of the class's systems.
        Returns {class: entry}."""
        import torch

        gpu = torch.cuda.get_device_name() + f"/{torch.cuda.get_device_properties(0).multi_processor_count}SM"
        shapes = batch_shapes(batch)
        plan = {}
        for c, mo, sub in batch.class_items(batch.items(sample_omegas, "system")):
            members = sorted(set(int(i) for i in sub.system.cpu().numpy()))
            key = batch_signature([shapes[i] for i in members], f"{precision}/class", gpu)

            def measure(bps: int, order: str, sub=sub, mo=mo) -> float:
                if batch.max_grid(precision, bps, mo) <= 0:
                    raise RuntimeError("launch shape not available")
                it = sub.reordered(order)
                batch.launch(it, precision, blocks_per_sm=bps, max_order=mo)  # warm-up
                best = float("inf")
                for _ in range(reps):
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    batch.launch(it, precision, blocks_per_sm=bps, max_order=mo)
                    e1.record()
                    torch.cuda.synchronize()
                    best = min(best, e0.elapsed_time(e1))
                return best

            plan[c] = self.select(key, measure, force)
        return plan


class ProductPathTuner(BatchTuner):
    """Chooses the FP32 product tiling (0 mma.sync, 1 tcgen05) per block order."""

    def __init__(self, cache_path: str | Path | None = None):
        super().__init__(cache_path, candidates=[(1, "mma.sync"), (1, "tcgen05")])

    def tune(self, system, omega, k_index, eta, precision: str = "mixed", reps: int = 2,
             force: bool = False) -> dict:
        """Times ``system.transmission(omega, k_index, eta, precision)`` with each
        tiling, keeps the faster for ``system.n`` and returns the entry
        (``path`` 0 or 1).  Orders above 128 have only mma.sync."""
        import torch

        from . import engine

        n = system.n
        if n > 128:
            engine.set_fp32_product_path(n, 0)
            return {"path": 0, "order": "mma.sync", "cached": False, "timings": {}}
        gpu = torch.cuda.get_device_name() + f"/{torch.cuda.get_device_properties(0).multi_processor_count}SM"
        key = batch_signature([(n, system.nl, system.nr, system.n_layers, 0, 0)], "fp32-product/" + precision, gpu)

        def measure(_bps: int, order: str) -> float:
            engine.set_fp32_product_path(n, 1 if order == "tcgen05" else 0)
            system.transmission(omega, k_index, eta, precision=precision)  # warm-up
            best = float("inf")
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                system.transmission(omega, k_index, eta, precision=precision)
                e1.record()
                torch.cuda.synchronize()
                best = min(best, e0.elapsed_time(e1))
            return best

        entry = self.select(key, measure, force)
        path = 1 if entry["order"] == "tcgen05" else 0
        engine.set_fp32_product_path(n, path)
        return dict(entry, path=path)
