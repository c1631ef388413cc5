"""k-space blocks built on the GPU against the host builder, and the batched
transmission through them against the general per-k path."""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

import negfpy_b200 as nb  # noqa: E402
from negfpy_b200 import workloads as W  # noqa: E402
from negfpy_b200.kspace import kspace_stack  # noqa: E402
from negfpy_b200.models import (MaterialKspaceParams, material_kspace_device, material_kspace_lead,  # noqa: E402
                                material_kspace_stack)
from negfpy_b200.types import DeviceKSpace, LeadKSpace  # noqa: E402


def _params(pin=0.0):
    p = W.spring_network(3, ny=2, nz=8, periodic_y=True, periodic_z=True)
    return MaterialKspaceParams(masses=p.masses, fc00_terms=p.fc00_terms, fc01_terms=p.fc01_terms,
                                dof_per_atom=3, onsite_pinning=pin)


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_blocks_match_host_builder():
    prm = _params(pin=0.3)
    kp = W.kgrid(4, 3)
    rng = np.random.default_rng(0)
    lm = rng.uniform(0.7, 1.3, size=(5, prm.n_atoms))
    host = material_kspace_stack(prm, kp, layer_masses=lm, n_layers=5)
    gpu = kspace_stack(prm, kp, n_layers=5, layer_masses=lm)
    for key in ("d00", "d01", "d10", "onsite", "coupling"):
        assert _rel(gpu[key].cpu().numpy(), host[key]) < 1e-14, key
    uni = kspace_stack(prm, kp, n_layers=5)
    assert uni["onsite"].shape[1] == 1 and _rel(uni["onsite"][:, 0].cpu().numpy(), host["d00"]) < 1e-14


def test_transmission_grid_fast_path_matches_general_path():
    prm = _params()
    lead, dev = material_kspace_lead(prm), material_kspace_device(6, prm)
    kp = W.kgrid(3, 2)
    wmax = W.estimate_omega_max(prm, nk=3, two_d=True)
    om = (np.arange(24) + 0.5) * (1.05 * wmax / 24)
    eta = 1e-6 * wmax * wmax
    fast = nb.transmission_grid(om, kp, dev, lead, lead, eta=eta)
    # wrappers without the builder attributes take the general (per-k host) path
    lead_g = LeadKSpace(blocks_builder=lambda k: lead.blocks(k))
    dev_g = DeviceKSpace(device_builder=lambda k: dev.device(k))
    slow = nb.transmission_grid(om, kp, dev_g, lead_g, lead_g, eta=eta)
    assert (fast["status"] == 0).all() and (slow["status"] == 0).all()
    # the two block builders agree to rounding (1e-16); T's conditioning lifts that
    # to ~1e-11 at some points, inside the 1e-10 parity bound against negfpy
    err = np.abs(fast["T"] - slow["T"]) / np.maximum(np.abs(slow["T"]), 1.0)
    assert float(err.max()) < 1e-10
