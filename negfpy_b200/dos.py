"""Drop-in lead surface DOS (negfpy ``core/dos.py:31-251``) on the GPU.

The DOS trace (omega/pi) Re Tr[i (g - g^H)] is the epilogue of the
Sancho-Rubio kernel, so the surface Green's function never leaves the GPU.
k lists run as one batch; the eta ladder re-launches only failed points.
"""

from __future__ import annotations

from typing import Iterable

import numpy as np
import torch

from . import _lib, engine
from .surface_gf import check_method, raise_for_status
from .types import resolve_lead_blocks


def _stack_leads(lead, kpoints):
    blocks = [resolve_lead_blocks(lead, k) for k in kpoints]
    d00 = np.stack([np.asarray(b.d00, dtype=np.complex128) for b in blocks])
    d01 = np.stack([np.asarray(b.d01, dtype=np.complex128) for b in blocks])
    d10 = None
    if all(b.d10 is not None for b in blocks):
        d10 = np.stack([np.asarray(b.d10, dtype=np.complex128) for b in blocks])
    elif any(b.d10 is not None for b in blocks):
        d10 = np.stack([np.asarray(b.d10 if b.d10 is not None else np.conj(b.d01).T, dtype=np.complex128)
                        for b in blocks])
    return d00, d01, d10


def _dos_batch(omegas, lead, kpoints, etas, normalize_per_mode):
    """DOS and status for points (omega_i, k_i, eta_i), one launch."""
    dev = _lib.require_cuda()
    d00, d01, d10 = _stack_leads(lead, kpoints)
    P = len(kpoints)
    om = torch.tensor(np.asarray(omegas, dtype=float), dtype=torch.float64, device=dev)
    et = torch.tensor(np.asarray(etas, dtype=float), dtype=torch.float64, device=dev)
    ki = torch.arange(P, dtype=torch.int32, device=dev)
    r = engine.sgf_sr(engine._c(d00), engine._c(d01), None if d10 is None else engine._c(d10), om, et, ki,
                      want_g=False, want_dos=True)
    dos = r["dos"].cpu().numpy()
    if normalize_per_mode:
        dos = dos / d00.shape[-1]
    return dos, r["status"].cpu().numpy()


def lead_surface_dos(omega: float, lead, eta: float = 1e-8, kpar=None, *, normalize_per_mode: bool = False,
                     surface_gf_method: str = "sancho_rubio") -> float:
    """Surface DOS at (omega, k) (negfpy ``core/dos.py:31-61``)."""
    if omega < 0.0:
        raise ValueError("omega must be non-negative.")
    check_method(surface_gf_method)
    d, st = _dos_batch([omega], lead, [kpar], [eta], normalize_per_mode)
    raise_for_status(int(st[0]))
    return float(d[0])


def lead_surface_dos_kavg(omega: float, lead, kpoints: list, eta: float = 1e-8, *, normalize_per_mode: bool = False,
                          surface_gf_method: str = "sancho_rubio") -> float:
    """k-averaged surface DOS (negfpy ``core/dos.py:64-88``)."""
    if len(kpoints) == 0:
        raise ValueError("kpoints must contain at least one k-point.")
    if omega < 0.0:
        raise ValueError("omega must be non-negative.")
    check_method(surface_gf_method)
    d, st = _dos_batch([omega] * len(kpoints), lead, kpoints, [eta] * len(kpoints), normalize_per_mode)
    for s in st:
        raise_for_status(int(s))
    return float(np.mean(d))


def lead_surface_dos_kavg_adaptive(omega: float, lead, kpoints: list, eta_values: tuple = (1e-8, 1e-7, 1e-6, 1e-5),
                                   min_success_fraction: float = 0.0, *, normalize_per_mode: bool = False,
                                   surface_gf_method: str = "sancho_rubio") -> tuple[float, dict]:
    """Per-k eta ladder for the DOS (negfpy ``core/dos.py:91-158``)."""
    if len(kpoints) == 0:
        raise ValueError("kpoints must contain at least one k-point.")
    if len(eta_values) == 0:
        raise ValueError("eta_values must contain at least one eta value.")
    if not (0.0 <= min_success_fraction <= 1.0):
        raise ValueError("min_success_fraction must be in [0, 1].")
    check_method(surface_gf_method)
    K = len(kpoints)
    accepted: dict[int, tuple[float, float]] = {}
    pending = list(range(K))
    for eta in eta_values:
        if not pending:
            break
        if omega < 0.0:  # the reference's ValueError is caught per point
            break
        d, st = _dos_batch([omega] * len(pending), lead, [kpoints[i] for i in pending], [eta] * len(pending),
                           normalize_per_mode)
        nxt = []
        for j, ki in enumerate(pending):
            if st[j] == _lib.OK and np.isfinite(d[j]):
                accepted[ki] = (float(d[j]), float(eta))
            else:
                nxt.append(ki)
        pending = nxt
    vals = [accepted[i][0] for i in range(K) if i in accepted]
    used = [accepted[i][1] for i in range(K) if i in accepted]
    n_success = len(vals)
    success_fraction = float(n_success / K)
    if n_success == 0:
        raise RuntimeError("No k-point converged for adaptive k-averaged DOS.")
    if success_fraction < min_success_fraction:
        raise RuntimeError(
            "Adaptive k-averaged DOS failed success-fraction threshold "
            f"(got {success_fraction:.3f}, required >= {min_success_fraction:.3f}).")
    info = {
        "n_total": int(K),
        "n_success": int(n_success),
        "n_failed": int(K - n_success),
        "success_fraction": success_fraction,
        "eta_histogram": {float(e): int(sum(1 for u in used if u == float(e))) for e in eta_values},
    }
    return float(np.mean(vals)), info


def lead_surface_dos_spectrum(omegas: Iterable[float], lead, *, kpoints: list | None = None, eta: float = 1e-8,
                              eta_values: tuple | None = None, min_success_fraction: float = 0.0,
                              normalize_per_mode: bool = False,
                              surface_gf_method: str = "sancho_rubio") -> np.ndarray:
    """DOS(omega) for one lead (negfpy ``core/dos.py:161-213``); the fixed-eta
    forms run the whole (omega, k) grid as one batch."""
    omega_arr = np.asarray(list(omegas), dtype=float)
    if omega_arr.ndim != 1 or omega_arr.size == 0:
        raise ValueError("omegas must be a non-empty 1D iterable.")
    check_method(surface_gf_method)
    if eta_values is not None and kpoints is not None:
        return np.array([lead_surface_dos_kavg_adaptive(float(w), lead, kpoints, eta_values, min_success_fraction,
                                                        normalize_per_mode=normalize_per_mode)[0]
                         for w in omega_arr])
    if np.any(omega_arr < 0.0):
        raise ValueError("omega must be non-negative.")
    ks = [None] if kpoints is None else list(kpoints)
    K = len(ks)
    om = np.repeat(omega_arr, K)
    kk = ks * omega_arr.size
    d, st = _dos_batch(om, lead, kk, [eta] * om.size, normalize_per_mode)
    for s in st:
        raise_for_status(int(s))
    return d.reshape(omega_arr.size, K).mean(axis=1)


def leads_surface_dos_spectrum(omegas: Iterable[float], lead_left, lead_right, *, kpoints: list | None = None,
                               eta: float = 1e-8, eta_values: tuple | None = None, min_success_fraction: float = 0.0,
                               normalize_per_mode: bool = False,
                               surface_gf_method: str = "sancho_rubio") -> dict:
    """DOS spectra of both leads (negfpy ``core/dos.py:216-251``)."""
    om = list(omegas)
    kw = dict(kpoints=kpoints, eta=eta, eta_values=eta_values, min_success_fraction=min_success_fraction,
              normalize_per_mode=normalize_per_mode, surface_gf_method=surface_gf_method)
    return {"left": lead_surface_dos_spectrum(om, lead_left, **kw),
            "right": lead_surface_dos_spectrum(om, lead_right, **kw)}
