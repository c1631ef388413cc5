"""k-space blocks of a force-constant model for all k at once on the GPU
(``negf_kspace_blocks_f64``), replacing the per-k Python phase sums and mass
weighting of negfpy ``models/material_kspace.py:99-195``.

``kspace_stack`` returns device-resident stacked blocks; ``stacked_system``
builds the ``engine.StackedSystem`` of a material lead / device / lead
problem directly from them (the fast path of ``spectrum.transmission_grid``).
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib, engine
from .models import MaterialKspaceParams, interface_terms, parse_ky_kz


def real_terms(*groups) -> bool:
    """True when every force-constant block is real (the kernel's operand type)."""
    return all(not np.iscomplexobj(v) or not np.any(np.imag(v)) for g in groups if g is not None for v in g.values())


def _phase_sum(terms: dict, kpts: torch.Tensor, wr: torch.Tensor, wc: torch.Tensor, pin: float) -> torch.Tensor:
    if not real_terms(terms):
        raise ValueError("negf_kspace_blocks_f64 takes real force-constant blocks; complex ones need the host builder")
    lib = _lib.load()
    dev = kpts.device
    keys = list(terms.keys())
    blocks = torch.as_tensor(np.stack([np.real(np.asarray(terms[k])).astype(float) for k in keys]),
                             device=dev).contiguous()
    shifts = torch.as_tensor(np.asarray(keys, dtype=float), device=dev).contiguous()
    K, n = kpts.shape[0], blocks.shape[-1]
    out = torch.empty((K, n, n), dtype=torch.complex128, device=dev)
    rc = lib.negf_kspace_blocks_f64(blocks.data_ptr(), shifts.data_ptr(), len(keys), kpts.data_ptr(), K, n,
                                    wr.data_ptr(), wc.data_ptr(), float(pin), out.data_ptr(), _lib.stream_handle())
    _lib.check(rc, "negf_kspace_blocks_f64")
    return out


def kspace_stack(params: MaterialKspaceParams, kpoints, n_layers: int | None = None, layer_masses=None,
                 scale2: float = 1.0) -> dict:
    """Lead blocks d00 / d01 / d10 ``[K, n, n]`` and, with ``n_layers``, device
    onsite ``[K, L|1, n, n]`` and coupling ``[K, L-1|1, n, n]`` (one layer when
    the layer masses are the model's), complex128 on the current GPU, every
    block divided by ``scale2``."""
    dev = _lib.require_cuda()
    kk = [parse_ky_kz(k) for k in kpoints]
    kpts = torch.as_tensor(np.asarray(kk, dtype=float).reshape(-1, 2), device=dev).contiguous()
    n = params.ndof
    w = torch.as_tensor(1.0 / np.sqrt(np.repeat(np.asarray(params.masses, dtype=float), params.dof_per_atom)),
                        device=dev) / np.sqrt(scale2)
    pin = float(params.onsite_pinning)
    out = {"d00": _phase_sum(params.fc00_terms, kpts, w, w, pin), "d01": _phase_sum(params.fc01_terms, kpts, w, w, 0.0)}
    if params.fc10_terms is None:
        out["d10"] = out["d01"].conj().transpose(-1, -2).contiguous()
    else:
        out["d10"] = _phase_sum(params.fc10_terms, kpts, w, w, 0.0)
    if n_layers is not None:
        if layer_masses is None:
            out["onsite"] = out["d00"][:, None]
            out["coupling"] = out["d01"][:, None]
        else:
            one = torch.ones(n, dtype=torch.float64, device=dev)
            phi00 = _phase_sum(params.fc00_terms, kpts, one, one, pin)
            phi01 = _phase_sum(params.fc01_terms, kpts, one, one, 0.0)
            lm = np.asarray(layer_masses, dtype=float)
            ms = torch.as_tensor(1.0 / np.sqrt(np.repeat(lm, params.dof_per_atom, axis=1)), device=dev) / np.sqrt(scale2)
            out["onsite"] = (ms[None, :, :, None] * phi00[:, None] * ms[None, :, None, :]).contiguous()
            out["coupling"] = (ms[None, :-1, :, None] * phi01[:, None] * ms[None, 1:, None, :]).contiguous()
    return out


def stacked_system(lead_params: MaterialKspaceParams, device_info: dict, kpoints) -> engine.StackedSystem:
    """StackedSystem of material lead | device | same lead with negfpy's default
    couplings (V_L = d10, V_R = d01) and contacts (the first / last layer)."""
    st = kspace_stack(lead_params, kpoints, device_info["n_layers"], device_info["layer_masses"])
    lead = (st["d00"], st["d01"], st["d10"])
    return engine.StackedSystem(lead, lead, st["onsite"].contiguous(), st["coupling"].contiguous(),
                                int(device_info["n_layers"]), st["d10"], st["d01"], True)


def interface_system(params: MaterialKspaceParams, device_info: dict, kpoints) -> engine.StackedSystem:
    """StackedSystem of the IFC transport set-up of ``models.interface_contacts``
    (negfpy ``workflows/ifc_bulk.py:690-742``) around a material device: all
    k blocks of both leads, the device and the couplings V_R = d01 of the
    right lead, V_L = V_R^H, built on the GPU."""
    st = kspace_stack(params, kpoints, device_info["n_layers"], device_info["layer_masses"])
    dev = st["d00"].device
    kk = [parse_ky_kz(k) for k in kpoints]
    kpts = torch.as_tensor(np.asarray(kk, dtype=float).reshape(-1, 2), device=dev).contiguous()
    w = torch.as_tensor(1.0 / np.sqrt(np.repeat(np.asarray(params.masses, dtype=float), params.dof_per_atom)),
                        device=dev)
    left_terms, right_terms = interface_terms(params)
    d01l = _phase_sum(left_terms, kpts, w, w, 0.0)
    d01r = _phase_sum(right_terms, kpts, w, w, 0.0)
    herm = lambda a: a.conj().transpose(-1, -2).contiguous()  # noqa: E731
    lead_l = (st["d00"], d01l, herm(d01l))
    lead_r = (st["d00"], d01r, herm(d01r))
    return engine.StackedSystem(lead_l, lead_r, st["onsite"].contiguous(), st["coupling"].contiguous(),
                                int(device_info["n_layers"]), herm(d01r), d01r, False)
