"""Batched (omega x k) transmission, DOS and kappa: the fast entry points.

``transmission_grid`` evaluates a whole omega grid times a k list in one
batched pass (the form negfpy's workflow builds from thousands of scalar
calls, ``workflows/ifc_bulk.py:951-1021, 1059-1288``); ``kappa_from_grid``
reduces it to kappa(T) on the GPU (``workflows/ifc_bulk.py:408-438``).
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib, engine
from .negf import point_system, stack_systems
from .surface_gf import check_method


def system_over_k(device, lead_left, lead_right, kpoints, eta_device=None, device_to_lead_left=None,
                  device_to_lead_right=None, contact_left_indices=None, contact_right_indices=None,
                  omega_scale=None) -> engine.StackedSystem:
    """Resolve and upload the blocks of every k once (omega-independent).

    Material lead / device / same lead with default couplings and contacts
    and no omega_scale: every k is built on the GPU (``kspace.stacked_system``)."""
    ks = [None] if kpoints is None else list(kpoints)
    fast = _material_fast_path(device, lead_left, lead_right, device_to_lead_left, device_to_lead_right,
                               contact_left_indices, contact_right_indices, omega_scale)
    if fast is not None:
        from .kspace import interface_system, stacked_system

        build = interface_system if fast[0] == "interface" else stacked_system
        return build(fast[1], fast[2], [() if k is None else k for k in ks])
    systems = [point_system(1.0, device, lead_left, lead_right, 1.0, eta_device, k, device_to_lead_left,
                            device_to_lead_right, contact_left_indices, contact_right_indices, omega_scale)
               for k in ks]
    sysobj, _ = stack_systems(systems)
    return sysobj


def _material_fast_path(device, lead_left, lead_right, vdl_left, vdl_right, idx_l, idx_r, omega_scale):
    """(kind, params, device info) when the GPU block builder covers the system:
    kind "material" for ``material_kspace_lead`` leads with the default
    couplings, "interface" for the four pieces of one ``interface_contacts``
    set-up; both around ``material_kspace_device`` of the same parameters,
    with default contacts, no omega scale and real force constants."""
    from .kspace import real_terms

    if any(x is not None for x in (idx_l, idx_r, omega_scale)):
        return None
    db = getattr(device, "device_builder", None)
    dp = getattr(db, "kspace_params", None)
    info = getattr(db, "kspace_device", None)
    if dp is None or info is None or not real_terms(dp.fc00_terms, dp.fc01_terms, dp.fc10_terms):
        return None
    if vdl_left is None and vdl_right is None:
        lb = getattr(getattr(lead_left, "blocks_builder", None), "kspace_params", None)
        rb = getattr(getattr(lead_right, "blocks_builder", None), "kspace_params", None)
        return ("material", dp, info) if lb is dp and rb is dp else None
    tags = [getattr(x, "kspace_interface", None) for x in (getattr(lead_left, "blocks_builder", None),
                                                          getattr(lead_right, "blocks_builder", None),
                                                          vdl_left, vdl_right)]
    if any(t is None for t in tags):
        return None
    token = tags[0][0]
    roles = ["left", "right", "vdl_left", "vdl_right"]
    if all(t[0] is token and t[1] is dp and t[2] == r for t, r in zip(tags, roles)):
        return "interface", dp, info
    return None


def grid_points(W: int, K: int, device=None):
    """omega-major point layout: p = w * K + k."""
    dev = device or _lib.require_cuda()
    w_idx = torch.arange(W, device=dev, dtype=torch.int64).repeat_interleave(K)
    k_idx = torch.arange(K, device=dev, dtype=torch.int32).repeat(W)
    return w_idx, k_idx


def transmission_grid(omegas, kpoints, device, lead_left, lead_right, eta: float = 1e-8,
                      eta_device: float | None = None, device_to_lead_left=None, device_to_lead_right=None,
                      contact_left_indices=None, contact_right_indices=None, surface_gf_method: str = "sancho_rubio",
                      omega_scale: float | None = None, tol: float = 1e-12, maxiter: int = 200,
                      precision: str = "f64") -> dict:
    """T[w, k] for every omega and k (numpy arrays ``T``, ``status``, ``iters_left``, ``iters_right``).

    Each entry equals ``negfpy.core.transmission(omegas[w], ..., kpar=kpoints[k])``.
    ``precision``: "f64"; "refined" (FP32 factors of the device solve refined
    to FP64 accuracy, FP64 re-solve of the points that fail; adds ``steps``
    and the count ``fallback``); "mixed" (unrefined FP32 sweep, about FP32
    accuracy; adds ``fallback``).
    """
    check_method(surface_gf_method)
    dev = _lib.require_cuda()
    om = np.asarray(omegas, dtype=float).ravel()
    sysobj = system_over_k(device, lead_left, lead_right, kpoints, eta_device, device_to_lead_left,
                           device_to_lead_right, contact_left_indices, contact_right_indices, omega_scale)
    s = 1.0 if omega_scale is None else float(omega_scale)
    eta_dev = float(eta if eta_device is None else eta_device)
    if eta_dev < 0.0:
        raise ValueError("eta_device must be non-negative.")
    K = sysobj.K
    w_idx, k_idx = grid_points(om.size, K, dev)
    om_t = torch.tensor(om / s, dtype=torch.float64, device=dev)[w_idx]
    P = om.size * K
    r = sysobj.transmission(om_t, k_idx, torch.full((P,), eta / s, dtype=torch.float64, device=dev),
                            torch.full((P,), eta_dev / s, dtype=torch.float64, device=dev), tol, maxiter,
                            precision=precision)
    out = {key: v.reshape(om.size, K).cpu().numpy() for key, v in r.items() if torch.is_tensor(v)}
    if precision != "f64":
        out["fallback"] = int(r["fallback"])
    return out


def kappa_from_grid(omegas, T_wk, temperatures, omega_unit_rad_s: float) -> np.ndarray:
    """kappa(T) from a [W, K] transmission table: k mean then the Bose-weighted trapezoid, on the GPU."""
    dev = _lib.require_cuda()
    om = torch.as_tensor(np.asarray(omegas, dtype=float), device=dev)
    T = torch.as_tensor(np.asarray(T_wk, dtype=float), device=dev)
    if T.dim() == 1:
        T = T[:, None]
    tbar = engine.kavg(T)
    return engine.kappa(om, tbar, temperatures, omega_unit_rad_s).cpu().numpy()


def thermal_conductance_from_spectrum(omegas, transmission_vals, temperatures, omega_unit_rad_s: float) -> np.ndarray:
    """negfpy ``workflows/ifc_bulk.py:408-438`` with an explicit rad/s unit factor.

    The reference converts its QE internal frequency unit with
    ``qe_omega_to_rad_s``; pass that factor as ``omega_unit_rad_s`` to get the
    same numbers.  Same validation: 1-D arrays of equal length, strictly
    increasing omega; temperatures <= 0 give 0.
    """
    om = np.asarray(omegas, dtype=float)
    tv = np.asarray(transmission_vals, dtype=float)
    if om.ndim != 1 or tv.ndim != 1 or om.size != tv.size:
        raise ValueError("omega_qe and transmission_vals must be 1D arrays of equal length.")
    if np.any(np.diff(om) <= 0.0):
        raise ValueError("omega_qe must be strictly increasing.")
    return kappa_from_grid(om, tv, np.asarray(temperatures, dtype=float), omega_unit_rad_s)
