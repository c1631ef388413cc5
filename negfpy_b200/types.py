"""Lead and device block containers for the batched phonon NEGF path.

These mirror negfpy's public data types (``core/types.py:16-86``) field for
field, with the same validation and error messages, so objects built for
negfpy can be handed to this package unchanged.  Every function in this
package also accepts negfpy's own instances: it only relies on the
attributes (``d00``/``d01``/``d10``, ``blocks(kpar)``, ``onsite_blocks``/
``coupling_blocks``, ``device(kpar)``), never on the class identity.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Callable

import numpy as np

Array = np.ndarray
KPar = tuple[float, ...] | None


@dataclass(frozen=True)
class LeadBlocks:
    """Periodic lead given by its principal-layer blocks (negfpy ``types.py:16-35``)."""

    d00: Array
    d01: Array
    d10: Array | None = None

    def __post_init__(self) -> None:
        if self.d00.ndim != 2 or self.d00.shape[0] != self.d00.shape[1]:
            raise ValueError("d00 must be a square 2D array.")
        if self.d01.ndim != 2:
            raise ValueError("d01 must be a 2D array.")
        if self.d01.shape != self.d00.shape:
            raise ValueError("d01 must have the same shape as d00.")
        if self.d10 is not None:
            if self.d10.ndim != 2:
                raise ValueError("d10 must be a 2D array when provided.")
            if self.d10.shape != self.d00.shape:
                raise ValueError("d10 must have the same shape as d00.")


@dataclass(frozen=True)
class LeadKSpace:
    """k_parallel-dependent lead provider (negfpy ``types.py:38-45``)."""

    blocks_builder: Callable[[KPar], tuple]

    def blocks(self, kpar: KPar = None) -> tuple:
        return self.blocks_builder(kpar)


@dataclass(frozen=True)
class Device1D:
    """Finite block-tridiagonal device (negfpy ``types.py:48-77``).

    All onsite and coupling blocks share one square shape; coupling block i
    sits at block position (i, i+1) and its conjugate transpose at (i+1, i).
    """

    onsite_blocks: list
    coupling_blocks: list

    def __post_init__(self) -> None:
        n_layers = len(self.onsite_blocks)
        if n_layers == 0:
            raise ValueError("Device must contain at least one principal layer.")
        if len(self.coupling_blocks) != n_layers - 1:
            raise ValueError("coupling_blocks length must be n_layers - 1.")
        first_shape = self.onsite_blocks[0].shape
        if len(first_shape) != 2 or first_shape[0] != first_shape[1]:
            raise ValueError("Each onsite block must be a square 2D array.")
        for block in self.onsite_blocks:
            if block.shape != first_shape:
                raise ValueError("All onsite blocks must share the same shape.")
        for block in self.coupling_blocks:
            if block.shape != first_shape:
                raise ValueError("All coupling blocks must match onsite block shape.")

    @property
    def n_layers(self) -> int:
        return len(self.onsite_blocks)

    @property
    def dof_per_layer(self) -> int:
        return int(self.onsite_blocks[0].shape[0])


@dataclass(frozen=True)
class DeviceKSpace:
    """k_parallel-dependent device provider (negfpy ``types.py:80-86``)."""

    device_builder: Callable[[KPar], Device1D]

    def device(self, kpar: KPar = None) -> Device1D:
        return self.device_builder(kpar)


def is_lead_blocks(obj) -> bool:
    return hasattr(obj, "d00") and hasattr(obj, "d01")


def is_device1d(obj) -> bool:
    return hasattr(obj, "onsite_blocks") and hasattr(obj, "coupling_blocks")


def resolve_lead_blocks(lead, kpar: KPar) -> LeadBlocks:
    """Blocks of a lead at one k (negfpy ``negf.py:22-32``, ``dos.py:18-28``)."""
    if is_lead_blocks(lead):
        return lead
    blocks = lead.blocks(kpar=kpar)
    if len(blocks) == 2:
        d00, d01 = blocks
        return LeadBlocks(d00=np.asarray(d00), d01=np.asarray(d01))
    if len(blocks) == 3:
        d00, d01, d10 = blocks
        return LeadBlocks(d00=np.asarray(d00), d01=np.asarray(d01), d10=np.asarray(d10))
    raise ValueError("LeadKSpace blocks_builder must return (d00,d01) or (d00,d01,d10).")


def resolve_device(device, kpar: KPar):
    """Device blocks at one k (negfpy ``negf.py:35-38``)."""
    if is_device1d(device):
        return device
    return device.device(kpar=kpar)
