"""Uneven batches: many independent systems of different block orders, layer
counts and k grids solved in ONE persistent launch (``negf_batch_transmission``).

Each system is a lead/device/lead problem of negfpy's path (``core/negf.py:306-357``
per (omega, k)); an item is (system, k index, omega).  The host

* uploads every system's stacked blocks once and writes the device-memory
  table of ``NegfBatchSystem`` records the kernel reads,
* orders the items (by default largest estimated cost first, so that the
  persistent blocks finish together),
* launches once, optionally inside a CUDA graph that is replayed for repeated
  solves of the same items,
* for ``precision="mixed_fallback"`` re-solves in FP64 the items whose FP32
  device sweep failed.  (The batch kernel has no iterative refinement: its
  mixed result carries FP32-level error; ``engine.StackedSystem`` with
  ``precision="refined"`` is the FP64-accurate reduced-precision solve.)

Launch shapes (blocks per SM) and the item order come from
``negfpy_b200.autotune``.  Two schedules: one launch over every item, or a
split schedule of one launch per padded-order class (the items whose
largest block order rounds up to the same multiple of 16), each class with
its own launch shape and item order; the tuner chooses per class and
between the schedules.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib, engine

PRECISIONS = {"f64": 0, "mixed": 1}


class NegfBatchSystem(C.Structure):
    """ctypes mirror of ``NegfBatchSystem`` (include/negf_b200.h)."""

    _fields_ = [
        ("n_dev", C.c_int), ("n_lead_l", C.c_int), ("n_lead_r", C.c_int), ("n_layers", C.c_int),
        ("n_k", C.c_int), ("same_leads", C.c_int),
        ("onsite", C.c_void_p), ("onsite_kstride", C.c_longlong), ("onsite_lstride", C.c_longlong),
        ("coupling", C.c_void_p), ("coupling_kstride", C.c_longlong), ("coupling_lstride", C.c_longlong),
        ("v_left", C.c_void_p), ("v_left_kstride", C.c_longlong),
        ("v_right", C.c_void_p), ("v_right_kstride", C.c_longlong),
        ("lead_l_h00", C.c_void_p), ("lead_l_h01", C.c_void_p), ("lead_l_h10", C.c_void_p),
        ("lead_l_kstride", C.c_longlong),
        ("lead_r_h00", C.c_void_p), ("lead_r_h01", C.c_void_p), ("lead_r_h10", C.c_void_p),
        ("lead_r_kstride", C.c_longlong),
        ("eta", C.c_double), ("eta_device", C.c_double),
    ]


def item_cost(n: int, nl: int, nr: int, L: int, same_leads: bool, sweeps: float = 18.0) -> float:
    """Estimated complex multiply-adds of one item: ``sweeps`` decimation sweeps
    of 7 order-m^3 steps per lead, 5 order-n^3 steps per layer."""
    c = sweeps * 7.0 * nl ** 3 + 5.0 * L * max(n, nl, nr) ** 3
    if not same_leads:
        c += sweeps * 7.0 * nr ** 3
    return c


def item_order(system: np.ndarray, cost: np.ndarray, order: str) -> np.ndarray:
    """Launch order of items (a permutation of their indices): "lpt" sorts by
    decreasing cost (stable), "system" keeps the given order, "interleave"
    takes one item of each system in turn."""
    P = system.size
    if order == "lpt":
        return np.argsort(-cost, kind="stable")
    if order == "system":
        return np.arange(P)
    if order == "interleave":
        rank = np.zeros(P, dtype=np.int64)
        for i in np.unique(system):
            idx = np.nonzero(system == i)[0]
            rank[idx] = np.arange(idx.size)
        return np.lexsort((system, rank))
    raise ValueError(f"unknown item order {order!r}; expected 'lpt', 'system' or 'interleave'")


def order_class(n: int, nl: int, nr: int) -> int:
    """Padded block order of a system (its largest order rounded up to 16):
    the class of its items in a split schedule."""
    return (max(n, nl, nr) + 15) // 16 * 16


@dataclass
class Items:
    system: torch.Tensor  # int32 [P], launch order
    k: torch.Tensor       # int32 [P]
    omega: torch.Tensor   # float64 [P]
    perm: torch.Tensor    # int64 [P]: launch position -> caller's item index
    cost: np.ndarray      # estimated cost per item, launch order

    def take(self, idx: np.ndarray) -> "Items":
        """The items at launch positions ``idx``, in that order."""
        sel = torch.as_tensor(idx, device=self.system.device)
        return Items(self.system[sel].contiguous(), self.k[sel].contiguous(), self.omega[sel].contiguous(),
                     self.perm[sel].contiguous(), self.cost[idx])

    def reordered(self, order: str) -> "Items":
        return self.take(item_order(self.system.cpu().numpy(), self.cost, order))


class UnevenBatch:
    """Device-resident systems of one uneven batch.

    ``systems``: objects with ``lead_l``/``lead_r`` dicts of ``d00/d01/d10``
    ``[K, m, m]``, ``onsite`` ``[K, L|1, n, n]``, ``coupling`` ``[K, L-1|1, n, n]``,
    ``n_layers``, ``eta``, optional ``eta_device``, ``vl``/``vr`` and
    ``same_leads`` (``workloads.Workload`` has them)."""

    def __init__(self, systems):
        dev = _lib.require_cuda()
        self.device = dev
        self.systems = []
        recs = []
        for w in systems:
            ll = tuple(engine._c(w.lead_l[x], dev) for x in ("d00", "d01", "d10"))
            same = bool(getattr(w, "same_leads", False) or w.lead_r is w.lead_l)
            lr = ll if same else tuple(engine._c(w.lead_r[x], dev) for x in ("d00", "d01", "d10"))
            s = engine.StackedSystem(ll, lr, engine._c(w.onsite, dev),
                                     None if w.coupling is None else engine._c(w.coupling, dev), int(w.n_layers),
                                     engine._c(w.vl if w.vl is not None else w.lead_l["d10"], dev),
                                     engine._c(w.vr if w.vr is not None else w.lead_r["d01"], dev), same)
            self.systems.append((s, float(w.eta), float(w.eta if w.eta_device is None else w.eta_device)))
            recs.append(self._record(s, float(w.eta), float(w.eta if w.eta_device is None else w.eta_device)))
        self.n_systems = len(recs)
        arr = (NegfBatchSystem * self.n_systems)(*recs)
        raw = torch.frombuffer(bytearray(C.string_at(C.addressof(arr), C.sizeof(arr))), dtype=torch.uint8)
        self.table = raw.to(dev)
        self.max_order = max(max(s.n, s.nl, s.nr) for s, _, _ in self.systems)
        self.sys_class = np.array([order_class(s.n, s.nl, s.nr) for s, _, _ in self.systems], dtype=np.int64)
        self.sys_order = np.array([max(s.n, s.nl, s.nr) for s, _, _ in self.systems], dtype=np.int64)
        self._graphs: dict = {}

    @staticmethod
    def _record(s: engine.StackedSystem, eta: float, eta_dev: float) -> NegfBatchSystem:
        K, Lo, n, _ = s.onsite.shape
        r = NegfBatchSystem()
        r.n_dev, r.n_lead_l, r.n_lead_r, r.n_layers, r.n_k = n, s.nl, s.nr, s.n_layers, K
        r.same_leads = 1 if s.same_leads else 0
        r.onsite, r.onsite_kstride, r.onsite_lstride = s.onsite.data_ptr(), (Lo * n * n if K > 1 else 0), (
            0 if Lo == 1 else n * n)
        if s.coupling is None or s.n_layers == 1:
            r.coupling, r.coupling_kstride, r.coupling_lstride = None, 0, 0
        else:
            Kc, Lc = s.coupling.shape[0], s.coupling.shape[1]
            r.coupling = s.coupling.data_ptr()
            r.coupling_kstride, r.coupling_lstride = (Lc * n * n if Kc > 1 else 0), (0 if Lc == 1 else n * n)
        r.v_left, r.v_left_kstride = s.vl.data_ptr(), (n * s.nl if s.vl.shape[0] > 1 else 0)
        r.v_right, r.v_right_kstride = s.vr.data_ptr(), (n * s.nr if s.vr.shape[0] > 1 else 0)
        for side, lead in (("l", s.lead_l), ("r", s.lead_r)):
            m = lead[0].shape[-1]
            setattr(r, f"lead_{side}_h00", lead[0].data_ptr())
            setattr(r, f"lead_{side}_h01", lead[1].data_ptr())
            setattr(r, f"lead_{side}_h10", None if lead[2] is None else lead[2].data_ptr())
            setattr(r, f"lead_{side}_kstride", m * m if lead[0].shape[0] > 1 else 0)
        r.eta, r.eta_device = eta, eta_dev
        return r

    # ------------------------------------------------------------------ items
    def items(self, omegas_per_system, order: str = "lpt") -> Items:
        """Items for every (system, omega, k) of the given omega arrays (one per
        system, its k grid in full), in ``order``: "lpt" (largest estimated cost
        first), "system" (system by system) or "interleave" (round-robin over
        systems)."""
        sys_i, k_i, om, cost = [], [], [], []
        for i, ((s, _, _), oms) in enumerate(zip(self.systems, omegas_per_system)):
            oms = np.asarray(oms, dtype=float).ravel()
            K = s.K
            sys_i.append(np.full(oms.size * K, i, dtype=np.int32))
            k_i.append(np.tile(np.arange(K, dtype=np.int32), oms.size))
            om.append(np.repeat(oms, K))
            cost.append(np.full(oms.size * K, item_cost(s.n, s.nl, s.nr, s.n_layers, s.same_leads)))
        sys_i, k_i, om, cost = (np.concatenate(x) for x in (sys_i, k_i, om, cost))
        perm = item_order(sys_i, cost, order)
        dev = self.device
        return Items(torch.as_tensor(sys_i[perm], device=dev), torch.as_tensor(k_i[perm], device=dev),
                     torch.as_tensor(om[perm], device=dev), torch.as_tensor(perm, device=dev), cost[perm])

    def class_items(self, it: Items, orders=None) -> list:
        """The items of each order class, as (class, max order, Items), classes
        ascending.  Within a class the items keep their order in ``it``, or are
        put in ``orders[class]`` ("lpt", "system" or "interleave")."""
        sys_np = it.system.cpu().numpy()
        cls = self.sys_class[sys_np]
        out = []
        for c in np.unique(cls):
            idx = np.nonzero(cls == c)[0]
            if orders is not None:
                idx = idx[item_order(sys_np[idx], it.cost[idx], orders[int(c)])]
            mo = int(self.sys_order[np.unique(sys_np[idx])].max())
            out.append((int(c), mo, it.take(idx)))
        return out

    # ----------------------------------------------------------------- launch
    def _buffers(self, P: int):
        dev = self.device
        return (torch.empty(P, dtype=torch.float64, device=dev), torch.empty(P, dtype=torch.int32, device=dev),
                torch.empty(P, dtype=torch.int32, device=dev))

    def max_grid(self, precision: str = "f64", blocks_per_sm: int = 1, max_order: int = 0) -> int:
        mo = int(max_order) or self.max_order
        return int(_lib.load().negf_batch_max_grid(mo, PRECISIONS[precision], int(blocks_per_sm)))

    def workspace_bytes(self, precision: str = "f64", blocks_per_sm: int = 1, grid: int = 0, max_order: int = 0):
        lib = _lib.load()
        mo = int(max_order) or self.max_order
        need = int(lib.negf_batch_workspace_bytes(mo, PRECISIONS[precision], int(blocks_per_sm), int(grid)))
        if need == 0:
            raise RuntimeError("negf_batch_workspace_bytes failed: " + lib.negf_last_error().decode())
        return need

    def launch(self, it: Items, precision: str = "f64", grid: int = 0, tol: float = 1e-12, maxiter: int = 200,
               out=None, stream=None, blocks_per_sm: int = 1, max_order: int = 0, ws=None):
        """One persistent launch over the items (launch order).  Returns
        (T, status, iters) in launch order.  ``max_order``: the largest block
        order among the items' systems (default: the batch's); ``ws``: a
        workspace of at least ``workspace_bytes`` (default: the cached one)."""
        lib = _lib.load()
        P = int(it.system.numel())
        T, st, iters = out if out is not None else self._buffers(P)
        prec = PRECISIONS[precision]
        mo = int(max_order) or self.max_order
        need = self.workspace_bytes(precision, blocks_per_sm, grid, mo)
        if ws is None:
            ws = engine._workspace(need, self.device, f"batch_{precision}")
        elif ws.numel() < need:
            raise ValueError(f"batch workspace of {ws.numel()} bytes; {need} needed")
        rc = lib.negf_batch_transmission(self.table.data_ptr(), self.n_systems, mo, it.system.data_ptr(),
                                         it.k.data_ptr(), it.omega.data_ptr(), P, float(tol), int(maxiter), prec,
                                         int(blocks_per_sm), int(grid), T.data_ptr(), st.data_ptr(), iters.data_ptr(), ws.data_ptr(),
                                         ws.numel(), _lib.stream_handle(stream))
        _lib.check(rc, "negf_batch_transmission")
        return T, st, iters

    def graph(self, it: Items, precision: str = "f64", grid: int = 0, tol: float = 1e-12, maxiter: int = 200,
              blocks_per_sm: int = 1):
        """A CUDA graph of the launch over ``it`` (counter reset + one kernel) and
        its output buffers; ``g.replay()`` re-solves the items."""
        P = int(it.system.numel())
        out = self._buffers(P)
        # the graph's own workspace, kept with the batch while the graph lives
        ws = torch.empty(self.workspace_bytes(precision, blocks_per_sm, grid), dtype=torch.uint8, device=self.device)
        # outside the capture: sets the kernel attributes
        self.launch(it, precision, grid, tol, maxiter, out, blocks_per_sm=blocks_per_sm, ws=ws)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.launch(it, precision, grid, tol, maxiter, out, blocks_per_sm=blocks_per_sm, ws=ws)
        torch.cuda.current_stream().wait_stream(s)
        self._graphs[id(g)] = ws
        return g, out

    # ------------------------------------------------------- split schedule
    def split_parts(self, it: Items, plan: dict | None = None) -> list:
        """The launches of the split schedule for ``it``: (class, max order,
        Items in the class's order, blocks per SM) per order class, from
        ``plan`` ({class: {"blocks_per_sm": b, "order": o}}; default one block
        per SM, largest cost first)."""
        plan = plan or {}
        orders = {int(c): plan.get(int(c), {}).get("order", "lpt") for c in np.unique(self.sys_class)}
        return [(c, mo, sub, int(plan.get(c, {}).get("blocks_per_sm", 1)))
                for c, mo, sub in self.class_items(it, orders)]

    def split_workspace_bytes(self, parts, precision: str = "f64") -> int:
        return max(self.workspace_bytes(precision, bps, 0, mo) for _, mo, _, bps in parts)

    def launch_split(self, parts, precision: str = "f64", tol: float = 1e-12, maxiter: int = 200, out=None,
                     ws=None):
        """The split schedule's launches, one after the other on the current
        stream.  Returns (T, status, iters) in the CALLER's item order (the
        class launches scatter their results through their ``perm``)."""
        P = sum(int(sub.system.numel()) for _, _, sub, _ in parts)
        T, st, iters = out if out is not None else self._buffers(P)
        for _, mo, sub, bps in parts:
            t, s_, i_ = self.launch(sub, precision, 0, tol, maxiter, blocks_per_sm=bps, max_order=mo, ws=ws)
            T[sub.perm] = t
            st[sub.perm] = s_
            iters[sub.perm] = i_
        return T, st, iters

    def graph_split(self, parts, precision: str = "f64", tol: float = 1e-12, maxiter: int = 200):
        """A CUDA graph of the split schedule (its own workspace, kept with the
        batch while the graph lives); ``g.replay()`` re-solves the items.
        Returns the graph and its (T, status, iters) in the caller's order."""
        P = sum(int(sub.system.numel()) for _, _, sub, _ in parts)
        out = self._buffers(P)
        ws = torch.empty(self.split_workspace_bytes(parts, precision), dtype=torch.uint8, device=self.device)
        self.launch_split(parts, precision, tol, maxiter, out, ws)  # kernel attributes, outside the capture
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.launch_split(parts, precision, tol, maxiter, out, ws)
        torch.cuda.current_stream().wait_stream(s)
        self._graphs[id(g)] = ws
        return g, out

    def release(self, g) -> None:
        """Drop the workspace kept for graph ``g`` (do not replay it afterwards)."""
        self._graphs.pop(id(g), None)

    def solve(self, it: Items, precision: str = "f64", grid: int = 0, tol: float = 1e-12,
              maxiter: int = 200, blocks_per_sm: int = 1) -> dict:
        """T, status and sweeps in the CALLER's item order.  ``precision``:
        "f64", "mixed", or "mixed_fallback" (mixed, then the FP64 re-solve of
        the items whose device sweep failed while their leads converged)."""
        if precision not in ("f64", "mixed", "mixed_fallback"):
            raise ValueError(f"unknown precision {precision!r}; expected 'f64', 'mixed' or 'mixed_fallback'")
        T, st, iters = self.launch(it, "f64" if precision == "f64" else "mixed", grid, tol, maxiter,
                                   blocks_per_sm=blocks_per_sm)
        n_fallback = 0
        if precision == "mixed_fallback":
            bad = (st == _lib.SINGULAR) | (st == _lib.NONFINITE)
            idx = torch.nonzero(bad).flatten()
            n_fallback = int(idx.numel())
            if n_fallback:
                sub = Items(it.system[idx].contiguous(), it.k[idx].contiguous(), it.omega[idx].contiguous(),
                            idx, it.cost[idx.cpu().numpy()])
                t2, s2, i2 = self.launch(sub, "f64", 0, tol, maxiter)
                T[idx], st[idx], iters[idx] = t2, s2, i2
        P = T.numel()
        out = {k: torch.empty_like(v) for k, v in (("T", T), ("status", st), ("iters", iters))}
        out["T"][it.perm] = T
        out["status"][it.perm] = st
        out["iters"][it.perm] = iters
        out["fallback"] = n_fallback
        out["items"] = P
        return out
