"""Landauer phonon heat current from transmission spectra (negfpy
``core/thermal_current.py``), with the spectral integral on the GPU
(``negf_heat_current_f64``) and the spectra from the batched device solve.

Same signatures, checks and error messages as negfpy; omegas in rad/s,
currents in W (W/m, W/m^2 for the per-length and per-area forms).
"""

from __future__ import annotations

from typing import Iterable

import numpy as np
import torch

from . import _lib
from .spectrum import transmission_grid
from .surface_gf import raise_for_status

HBAR = 1.054_571_817e-34  # J*s
KB = 1.380_649e-23  # J/K


def _to_1d_array(values: Iterable[float], name: str) -> np.ndarray:
    """negfpy ``core/thermal_current.py:20-28``."""
    arr = np.asarray(list(values), dtype=float)
    if arr.ndim != 1:
        raise ValueError(f"{name} must be 1D.")
    if arr.size < 2:
        raise ValueError(f"{name} must contain at least two points.")
    if np.any(np.diff(arr) <= 0.0):
        raise ValueError(f"{name} must be strictly increasing.")
    return arr


def heat_current_spectra(omegas, transmission_rows, temp_left: float, temp_right: float) -> np.ndarray:
    """Heat current of each row of ``transmission_rows`` [n_spectra, n_omega]
    on one omega grid (rad/s), in one launch."""
    omega = _to_1d_array(omegas, "omegas")
    rows = np.atleast_2d(np.asarray(transmission_rows, dtype=float))
    if rows.shape[1] != omega.size:
        raise ValueError("transmission_vals must have the same length as omegas.")
    if temp_left <= 0.0 or temp_right <= 0.0:
        raise ValueError("Temperatures must be positive in Kelvin.")
    dev = _lib.require_cuda()
    lib = _lib.load()
    om = torch.as_tensor(omega, device=dev)
    t = torch.as_tensor(np.ascontiguousarray(rows), device=dev)
    out = torch.empty(rows.shape[0], dtype=torch.float64, device=dev)
    _lib.check(lib.negf_heat_current_f64(om.data_ptr(), t.data_ptr(), omega.size, rows.shape[0], float(temp_left),
                                         float(temp_right), out.data_ptr(), _lib.stream_handle()),
               "negf_heat_current_f64")
    return out.cpu().numpy()


def heat_current_from_spectrum(omegas: Iterable[float], transmission_vals: Iterable[float], temp_left: float,
                               temp_right: float) -> float:
    """Phonon heat current (W) from T(omega) by the Landauer formula
    (negfpy ``core/thermal_current.py:50-67``); omegas in rad/s."""
    omega = _to_1d_array(omegas, "omegas")
    tvals = np.asarray(list(transmission_vals), dtype=float)
    if tvals.shape != omega.shape:
        raise ValueError("transmission_vals must have the same length as omegas.")
    return float(heat_current_spectra(omega, tvals[None, :], temp_left, temp_right)[0])


def _spectrum(omega, device, lead_left, lead_right, kpoints, eta) -> np.ndarray:
    res = transmission_grid(omega, kpoints, device, lead_left, lead_right, eta=eta)
    bad = np.flatnonzero(res["status"].ravel() != _lib.OK)
    if bad.size:
        raise_for_status(int(res["status"].ravel()[bad[0]]))
    return res["T"].mean(axis=1)


def heat_current_1d(omegas: Iterable[float], device, lead_left, lead_right, temp_left: float, temp_right: float,
                    eta: float = 1e-8) -> float:
    """1D phonon heat current (W) (negfpy ``core/thermal_current.py:70-99``)."""
    omega = _to_1d_array(omegas, "omegas")
    tvals = _spectrum(omega, device, lead_left, lead_right, None, eta)
    return heat_current_from_spectrum(omega, tvals, temp_left, temp_right)


def heat_current_per_length_2d(omegas: Iterable[float], device, lead_left, lead_right, kpoints,
                               transverse_length: float, temp_left: float, temp_right: float,
                               eta: float = 1e-8) -> float:
    """2D heat current per transverse length (W/m) (negfpy ``core/thermal_current.py:102-137``)."""
    if transverse_length <= 0.0:
        raise ValueError("transverse_length must be positive.")
    omega = _to_1d_array(omegas, "omegas")
    tavg = _spectrum(omega, device, lead_left, lead_right, kpoints, eta)
    return float(heat_current_from_spectrum(omega, tavg, temp_left, temp_right) / transverse_length)


def heat_current_density_3d(omegas: Iterable[float], device, lead_left, lead_right, kpoints, transverse_area: float,
                            temp_left: float, temp_right: float, eta: float = 1e-8) -> float:
    """3D heat current per transverse area (W/m^2) (negfpy ``core/thermal_current.py:140-175``)."""
    if transverse_area <= 0.0:
        raise ValueError("transverse_area must be positive.")
    omega = _to_1d_array(omegas, "omegas")
    tavg = _spectrum(omega, device, lead_left, lead_right, kpoints, eta)
    return float(heat_current_from_spectrum(omega, tavg, temp_left, temp_right) / transverse_area)


def transverse_length_from_vector(transverse_vec: Iterable[float], transport_dir: Iterable[float]) -> float:
    """Transverse periodic length orthogonal to transport (negfpy ``core/thermal_current.py:178-198``)."""
    t = np.asarray(list(transverse_vec), dtype=float)
    e = np.asarray(list(transport_dir), dtype=float)
    if t.ndim != 1 or e.ndim != 1 or t.shape != e.shape:
        raise ValueError("transverse_vec and transport_dir must be 1D with the same size.")
    en = np.linalg.norm(e)
    if en == 0.0:
        raise ValueError("transport_dir must be non-zero.")
    ehat = e / en
    t_perp = t - np.dot(t, ehat) * ehat
    length = float(np.linalg.norm(t_perp))
    if length == 0.0:
        raise ValueError("transverse_vec has zero component orthogonal to transport_dir.")
    return length
