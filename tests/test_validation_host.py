"""Argument checks of the DOS, k-mean and block-container APIs, with
negfpy's messages (core/dos.py:47-176, core/negf.py:377-433,
core/types.py:25-68).  Every check runs on the host before any launch."""

from __future__ import annotations

import numpy as np
import pytest

import negfpy_b200 as nb
from negfpy_b200.models import ChainParams, device_perfect_chain, lead_blocks


@pytest.fixture(scope="module")
def chain():
    p = ChainParams(1.0, 1.0)
    return device_perfect_chain(4, p), lead_blocks(p)


def test_dos_arguments(chain):
    _, lead = chain
    with pytest.raises(ValueError, match="omega must be non-negative"):
        nb.lead_surface_dos(-0.1, lead)
    with pytest.raises(ValueError, match="kpoints must contain at least one k-point"):
        nb.lead_surface_dos_kavg(0.5, lead, [])
    with pytest.raises(ValueError, match="kpoints must contain at least one k-point"):
        nb.lead_surface_dos_kavg_adaptive(0.5, lead, [])
    with pytest.raises(ValueError, match="eta_values must contain at least one eta value"):
        nb.lead_surface_dos_kavg_adaptive(0.5, lead, [()], ())
    with pytest.raises(ValueError, match=r"min_success_fraction must be in \[0, 1\]"):
        nb.lead_surface_dos_kavg_adaptive(0.5, lead, [()], (1e-6,), 1.5)
    with pytest.raises(ValueError, match="omegas must be a non-empty 1D iterable"):
        nb.lead_surface_dos_spectrum([], lead)
    with pytest.raises(ValueError, match="omegas must be a non-empty 1D iterable"):
        nb.lead_surface_dos_spectrum(np.ones((2, 2)), lead)


def test_kavg_arguments(chain):
    dev, lead = chain
    with pytest.raises(ValueError, match="kpoints must contain at least one k-point"):
        nb.transmission_kavg(0.5, dev, lead, lead, kpoints=[])
    with pytest.raises(ValueError, match="nonnegative_tolerance must be non-negative"):
        nb.transmission_kavg_adaptive(0.5, dev, lead, lead, kpoints=[()], nonnegative_tolerance=-1.0)
    with pytest.raises(ValueError, match="max_channel_factor must be positive"):
        nb.transmission_kavg_adaptive_global_eta(0.5, dev, lead, lead, kpoints=[()], max_channel_factor=0.0)


def test_block_containers():
    one = np.ones((2, 2), dtype=complex)
    with pytest.raises(ValueError, match="d00 must be a square 2D array"):
        nb.LeadBlocks(d00=np.ones((2, 3)), d01=one)
    with pytest.raises(ValueError, match="d01 must have the same shape as d00"):
        nb.LeadBlocks(d00=one, d01=np.ones((3, 3)))
    with pytest.raises(ValueError, match="d10 must have the same shape as d00"):
        nb.LeadBlocks(d00=one, d01=one, d10=np.ones((3, 3)))
    with pytest.raises(ValueError, match="Device must contain at least one principal layer"):
        nb.Device1D(onsite_blocks=[], coupling_blocks=[])
    with pytest.raises(ValueError, match="coupling_blocks length must be n_layers - 1"):
        nb.Device1D(onsite_blocks=[one, one], coupling_blocks=[])
    with pytest.raises(ValueError, match="All onsite blocks must share the same shape"):
        nb.Device1D(onsite_blocks=[one, np.ones((3, 3))], coupling_blocks=[one])
