"""Full device Green's function on the GPU against negfpy's
device_green_function (tests/golden/green.npz): G, Sigma_L, Sigma_R to 1e-10
of their largest entry."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import negfpy_b200 as nb  # noqa: E402
from negfpy_b200 import workloads as W  # noqa: E402

TOL = 1e-10


@pytest.fixture(scope="module")
def green():
    return np.load(Path(__file__).parent / "golden" / "green.npz")


def _check(got, green, key):
    for part, name in zip(got, ("G", "SL", "SR")):
        ref = green[f"{key}_{name}"]
        assert part.shape == ref.shape
        err = float(np.abs(part - ref).max() / np.abs(ref).max())
        assert err <= TOL, (key, name, err)


def test_chain(green):
    p = nb.ChainParams(1.0, 1.0)
    lead = nb.lead_blocks(p)
    _check(nb.device_green_function(1.1, nb.device_perfect_chain(6, p), lead, lead, eta=1e-8), green, "chain")


def test_rectangular_contacts(green):
    lead = nb.LeadBlocks(d00=np.array([[2.0]], dtype=complex), d01=np.array([[-1.0]], dtype=complex))
    on = [np.diag([2.0, 100.0]).astype(complex) for _ in range(4)]
    cp = [np.diag([-1.0, 0.0]).astype(complex) for _ in range(3)]
    got = nb.device_green_function(1.0, nb.Device1D(on, cp), lead, lead, eta=1e-8,
                                   device_to_lead_left=np.array([[-1.0]]), device_to_lead_right=np.array([[-1.0]]),
                                   contact_left_indices=[0], contact_right_indices=[6])
    _check(got, green, "rect")


def test_multidof_with_device_eta(green):
    # negfpy's MultiDofCellParams(masses=ones(2), fc00=2 I6, fc01=-I6): unit masses, D = Phi
    md = np.eye(6)
    lead = nb.LeadBlocks(d00=2.0 * md, d01=-md)
    got = nb.device_green_function(0.7, nb.Device1D([2.0 * md] * 5, [-md] * 4), lead, lead, eta=1e-7,
                                   eta_device=2e-7)
    _check(got, green, "md")


def test_slab_with_omega_scale(green):
    wl = W.slab_workload()
    ki = int(green["slab_k"])
    lb = nb.LeadBlocks(d00=wl.lead_l["d00"][ki], d01=wl.lead_l["d01"][ki], d10=wl.lead_l["d10"][ki])
    dv = nb.Device1D(onsite_blocks=[wl.onsite[ki, 0]] * 3, coupling_blocks=[wl.coupling[ki, 0]] * 2)
    got = nb.device_green_function(float(green["slab_omega"]), dv, lb, lb, eta=float(green["slab_eta"]),
                                   omega_scale=1.3)
    _check(got, green, "slab")
