"""Full counting statistics of coherent phonon heat transport (negfpy
``core/fcs.py``): the first two cumulants of the heat current from a
transmission spectrum or from k-resolved transmission moments, with the
moments and the spectral integrals on the GPU (``negf_kmoments_f64``,
``negf_fcs_cumulants_f64``).  Same signatures, checks and messages as negfpy;
omegas in rad/s.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Iterable

import numpy as np
import torch

from . import _lib


@dataclass(frozen=True)
class HeatCurrentCumulants:
    """First and second cumulants of heat current (per unit time)."""

    c1_j_per_s: float
    c2_j2_per_s: float


@dataclass(frozen=True)
class HeatCurrentUncertainty:
    """Finite-time uncertainty derived from the second cumulant."""

    measurement_time_s: float
    std_current_j_per_s: float
    variance_energy_j2: float
    std_energy_j: float


def _to_1d_array(values: Iterable[float], name: str) -> np.ndarray:
    """negfpy ``core/fcs.py:38-46``."""
    arr = np.asarray(list(values), dtype=float)
    if arr.ndim != 1:
        raise ValueError(f"{name} must be 1D.")
    if arr.size < 2:
        raise ValueError(f"{name} must contain at least two points.")
    if np.any(np.diff(arr) <= 0.0):
        raise ValueError(f"{name} must be strictly increasing.")
    return arr


def _cumulants(omega: np.ndarray, t1, t2, temp_left_k: float, temp_right_k: float) -> HeatCurrentCumulants:
    if temp_left_k <= 0.0 or temp_right_k <= 0.0:
        raise ValueError("Temperature must be positive in Kelvin.")
    dev = _lib.require_cuda()
    lib = _lib.load()
    om = torch.as_tensor(omega, device=dev)
    a = torch.as_tensor(t1, device=dev, dtype=torch.float64).contiguous()
    b = torch.as_tensor(t2, device=dev, dtype=torch.float64).contiguous()
    out = torch.empty(2, dtype=torch.float64, device=dev)
    _lib.check(lib.negf_fcs_cumulants_f64(om.data_ptr(), a.data_ptr(), b.data_ptr(), omega.size, float(temp_left_k),
                                          float(temp_right_k), out.data_ptr(), _lib.stream_handle()),
               "negf_fcs_cumulants_f64")
    c1, c2 = out.cpu().tolist()
    return HeatCurrentCumulants(c1_j_per_s=float(c1), c2_j2_per_s=float(c2))


def heat_current_cumulants_from_spectrum(omega_rad_s: Iterable[float], transmission_vals: Iterable[float],
                                         temp_left_k: float, temp_right_k: float) -> HeatCurrentCumulants:
    """C1 (J/s) and C2 (J^2/s) from T(omega) (negfpy ``core/fcs.py:85-116``)."""
    omega = _to_1d_array(omega_rad_s, "omega_rad_s")
    t = np.asarray(list(transmission_vals), dtype=float)
    if t.shape != omega.shape:
        raise ValueError("transmission_vals must have the same length as omega_rad_s.")
    if np.any(t < 0.0):
        raise ValueError("transmission_vals must be non-negative.")
    return _cumulants(omega, t, t * t, temp_left_k, temp_right_k)


def heat_current_cumulants_from_k_moments(omega_rad_s: Iterable[float], t_mean_vs_omega: Iterable[float],
                                          t2_mean_vs_omega: Iterable[float], temp_left_k: float,
                                          temp_right_k: float) -> HeatCurrentCumulants:
    """C1 and C2 from <T>_k and <T^2>_k (negfpy ``core/fcs.py:119-150``)."""
    omega = _to_1d_array(omega_rad_s, "omega_rad_s")
    t1 = np.asarray(list(t_mean_vs_omega), dtype=float)
    t2 = np.asarray(list(t2_mean_vs_omega), dtype=float)
    if t1.shape != omega.shape or t2.shape != omega.shape:
        raise ValueError("t_mean_vs_omega and t2_mean_vs_omega must match omega_rad_s shape.")
    if np.any(t1 < 0.0) or np.any(t2 < 0.0):
        raise ValueError("Transmission moments must be non-negative.")
    return _cumulants(omega, t1, t2, temp_left_k, temp_right_k)


def k_moments(t_wk) -> tuple[torch.Tensor, torch.Tensor]:
    """(<T>_k, <T^2>_k) per omega of an omega-major [W, K] table, on the GPU."""
    dev = _lib.require_cuda()
    lib = _lib.load()
    T = torch.as_tensor(t_wk, device=dev, dtype=torch.float64).contiguous()
    if T.dim() == 1:
        T = T[:, None]
    W, K = T.shape
    t1 = torch.empty(W, dtype=torch.float64, device=dev)
    t2 = torch.empty(W, dtype=torch.float64, device=dev)
    _lib.check(lib.negf_kmoments_f64(T.data_ptr(), W, K, t1.data_ptr(), t2.data_ptr(), _lib.stream_handle()),
               "negf_kmoments_f64")
    return t1, t2


def heat_current_cumulants_from_grid(omega_rad_s, t_wk, temp_left_k: float, temp_right_k: float) -> HeatCurrentCumulants:
    """C1 and C2 from a k-resolved [W, K] table (the k moments of negfpy's
    workflow, ``workflows/ifc_bulk.py:1690-1784``), moments and integrals on the GPU."""
    omega = _to_1d_array(omega_rad_s, "omega_rad_s")
    t1, t2 = k_moments(t_wk)
    if t1.numel() != omega.size:
        raise ValueError("t_mean_vs_omega and t2_mean_vs_omega must match omega_rad_s shape.")
    if bool((t1 < 0).any()) or bool((t2 < 0).any()):
        raise ValueError("Transmission moments must be non-negative.")
    return _cumulants(omega, t1, t2, temp_left_k, temp_right_k)


def heat_current_uncertainty(cumulants: HeatCurrentCumulants, *, measurement_time_s: float) -> HeatCurrentUncertainty:
    """Finite-time uncertainty from C2 (negfpy ``core/fcs.py:153-171``)."""
    tau = float(measurement_time_s)
    if tau <= 0.0:
        raise ValueError("measurement_time_s must be positive.")
    var_e = float(cumulants.c2_j2_per_s * tau)
    std_e = float(np.sqrt(max(var_e, 0.0)))
    std_j = float(np.sqrt(max(cumulants.c2_j2_per_s / tau, 0.0)))
    return HeatCurrentUncertainty(measurement_time_s=tau, std_current_j_per_s=std_j, variance_energy_j2=var_e,
                                  std_energy_j=std_e)
