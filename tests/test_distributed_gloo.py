"""Multi-rank sharding on CPU: two Gloo ranks, oracle-computed shards.

The GPU solve is replaced by the CPU oracle here (test infrastructure only);
what is checked is the sharding and the all-gather that assemble the full
spectrum, and that kappa from the gathered table equals the serial one.
"""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from negfpy_b200.distributed import gather_rows, omega_shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _chain_T(omegas):
    from oracle import negf_oracle as O

    lead = (np.array([[2.0]]), np.array([[-1.0]]), None)
    return np.array([[O.transmission_point(float(w), [np.array([[2.0]])] * 6, [np.array([[-1.0]])] * 5, lead, lead,
                                           eta=1e-8)] for w in omegas])


def _worker(rank, world, port, omegas, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        shard = omega_shard(len(omegas), rank, world)
        local = torch.as_tensor(_chain_T(omegas[shard]))
        full = gather_rows(local, len(omegas))
        np.save(os.path.join(out_dir, f"full_{rank}.npy"), full.numpy())
    finally:
        dist.destroy_process_group()


def test_omega_shard_partitions_the_grid():
    for n, world in ((17, 2), (16, 4), (3, 8)):
        parts = [omega_shard(n, r, world) for r in range(world)]
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(n))
        sizes = [p.size for p in parts]
        assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        omega_shard(4, 2, 2)


def test_two_gloo_ranks_gather_the_serial_spectrum(tmp_path):
    from oracle import negf_oracle as O

    omegas = (np.arange(13, dtype=float) + 0.5) * (2.0 / 13)
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), omegas, str(tmp_path)), nprocs=world, join=True)
    serial = _chain_T(omegas)
    for r in range(world):
        full = np.load(tmp_path / f"full_{r}.npy")
        assert np.array_equal(full, serial)
    unit = 2 * np.pi * 15e12 / 2.0
    k_full = O.thermal_conductance(omegas, full[:, 0], [300.0], unit)
    k_serial = O.thermal_conductance(omegas, serial[:, 0], [300.0], unit)
    assert np.array_equal(k_full, k_serial)


def _grad_worker(rank, world, port, omegas, weights, out_dir):
    """Fake local solve: value sum_w w f(w), gradient sum_w w df/dp, on CPU."""
    from negfpy_b200.distributed import sharded_weighted_sum

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        def local(om, w):
            f = np.sin(om) ** 2
            g = np.stack([np.cos(om) * w, om * w]).sum(axis=1)
            return torch.tensor([float((w * f).sum())], dtype=torch.float64), torch.as_tensor(g)

        k, g = sharded_weighted_sum(local, omegas, weights)
        np.save(os.path.join(out_dir, f"kg_{rank}.npy"), np.concatenate([k.numpy(), g.numpy()]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_kappa_and_gradient(tmp_path):
    """The sharded weighted sum with global trapezoid weights equals the serial one."""
    from negfpy_b200.adjoint import kappa_weights

    omegas = (np.arange(17, dtype=float) + 1.0) * 0.11
    weights = kappa_weights(torch.as_tensor(omegas), 300.0, 2 * np.pi * 15e12 / 2.0).numpy()
    world = 2
    mp.spawn(_grad_worker, args=(world, _free_port(), omegas, weights, str(tmp_path)), nprocs=world, join=True)
    serial = np.concatenate([[float((weights * np.sin(omegas) ** 2).sum())],
                             [float((np.cos(omegas) * weights).sum()), float((omegas * weights).sum())]])
    for r in range(world):
        got = np.load(tmp_path / f"kg_{r}.npy")
        np.testing.assert_allclose(got, serial, rtol=1e-13, atol=0)
