"""Sharding of an (omega x k) grid over ranks, one process per GPU.

Every (omega, k) point is independent (negfpy's own task farm is over omega,
``workflows/ifc_bulk.py:1212-1253``), so rank r of N takes the omegas
r, r+N, r+2N, ... with all k.  The strided split balances the work: cost
varies smoothly with omega (decimation sweeps, band edges), so contiguous
blocks would not.  The data path has no collective; one all-gather of the
per-rank T rows (a few KB to MB) assembles the spectrum where a caller wants
it (kappa, output files).  Works with any torch.distributed backend: NCCL
tensors on the rank's GPU, Gloo tensors on the CPU.
"""

from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist


def omega_shard(n_omega: int, rank: int, world: int) -> np.ndarray:
    """Omega indices of this rank (strided)."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError("rank must lie in [0, world)")
    return np.arange(rank, n_omega, world, dtype=np.int64)


def gather_rows(local: torch.Tensor, n_omega: int, group=None) -> torch.Tensor:
    """Assemble the full ``[n_omega, ...]`` table from every rank's strided rows.

    ``local`` holds this rank's rows in shard order (``omega_shard``).  All
    ranks must call it (one all-gather; shards are padded to equal length).
    """
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    per = (n_omega + world - 1) // world
    pad = torch.zeros((per,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    out = torch.empty((n_omega,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    for r in range(world):
        idx = omega_shard(n_omega, r, world)
        out[torch.as_tensor(idx, device=local.device)] = parts[r][: idx.size]
    del rank
    return out


def transmission_grid_sharded(omegas, kpoints, device, lead_left, lead_right, group=None, **kwargs) -> dict:
    """``transmission_grid`` over this rank's omega shard, gathered on every rank.

    Returns ``T`` and ``status`` for the whole grid (numpy) plus this rank's
    ``shard``.  Each rank computes on its current CUDA device.
    """
    from .spectrum import transmission_grid

    om = np.asarray(omegas, dtype=float)
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    shard = omega_shard(om.size, rank, world)
    res = transmission_grid(om[shard], kpoints, device, lead_left, lead_right, **kwargs)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    T = gather_rows(torch.as_tensor(res["T"], device=dev), om.size, group)
    st = gather_rows(torch.as_tensor(res["status"].astype(np.int32), device=dev), om.size, group)
    return {"T": T.cpu().numpy(), "status": st.cpu().numpy(), "shard": shard}


def sharded_weighted_sum(local_fn, omegas, weights, group=None):
    """sum_w weights[w] f(w) and its parameter gradients over the ranks.

    Every rank evaluates ``local_fn(omegas[shard], weights[shard])`` ->
    ``(value, *grads)`` (tensors) on its strided omega shard with the GLOBAL
    weights restricted to it (a trapezoid weight depends on both
    neighbours, so the shard must not re-derive them), then one all-reduce
    (sum) per output combines the ranks.  All ranks must call it."""
    om = np.asarray(omegas, dtype=float)
    w = np.asarray(weights, dtype=float)
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    shard = omega_shard(om.size, rank, world)
    outs = [torch.as_tensor(o).clone() for o in local_fn(om[shard], w[shard])]
    for o in outs:
        dist.all_reduce(o, op=dist.ReduceOp.SUM, group=group)
    return tuple(outs)


def hetero_kappa_grad_sharded(model, kpoints, omegas, eta, theta, masses=None, temperature=300.0,
                              omega_unit_rad_s=1.0, group=None):
    """kappa, dkappa/dtheta and dkappa/dmasses of a heterojunction with the
    omega grid sharded over the ranks (one adjoint launch per rank, one
    all-reduce of kappa and of each gradient: 2000 + 720 doubles for the
    differentiation workload).  Each rank computes on its current CUDA device."""
    from .adjoint import HeteroKappaProblem, kappa_weights

    om = np.asarray(omegas, dtype=float)
    w_all = kappa_weights(torch.as_tensor(om), temperature, omega_unit_rad_s).numpy()

    def local(om_s, w_s):
        pr = HeteroKappaProblem(model, kpoints, om_s, eta, temperature, omega_unit_rad_s,
                                w_kappa=torch.as_tensor(w_s))
        k, g_th, g_m = pr.kappa_and_grad(theta, masses)
        return k.reshape(1), g_th, g_m

    k, g_th, g_m = sharded_weighted_sum(local, om, w_all, group)
    return k[0], g_th, g_m
