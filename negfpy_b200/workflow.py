"""The workflow's transmission stage as batched GPU work (negfpy
``workflows/ifc_bulk.py:1059-1288``, ``_run_transmission``).

negfpy runs one task per omega in a thread or process pool, and each task
calls ``transmission_kavg_adaptive`` (per-k eta ladder), ``..._global_eta``
(one eta per omega) or the global form with the fixed eta, over the low or
the high k mesh of that omega.  Here the blocks of both meshes are uploaded
once, and every ladder rung is ONE launch over all pending (omega, k) points
of all omegas, each point with its own eta.  The acceptance tests, the
statistics, the eta records, the failure records, the rejected lists and the
post-processing of the values are negfpy's.

The ``solver.parallel`` settings are parsed and reported as negfpy reports
them; they do not change the execution (there is no pool).  The surface GF
method must be Sancho-Rubio (``NotImplementedError`` otherwise; negfpy's
workflow default is ``generalized_eigen_svd``, which is the oracle here).
"""

from __future__ import annotations

import os
from typing import Any

import numpy as np
import torch

from . import _lib
from .models import interface_contacts
from .negf import _check_adaptive_args, _classify, _prepare_ladder_systems, stack_systems
from .spectrum import _material_fast_path
from .surface_gf import check_method

# negfpy's name for the IFC transport set-up (workflows/ifc_bulk.py:690-742).
_build_interface_contacts = interface_contacts

# CODATA 2018 constants, as negfpy modeling/units.py:8-16.
RYDBERG_J = 2.1798723611035e-18
BOHR_M = 5.29177210903e-11
ELECTRON_MASS_KG = 9.1093837015e-31
QE_RY_MASS_UNIT_KG = 2.0 * ELECTRON_MASS_KG
SPEED_OF_LIGHT_CM_S = 2.99792458e10
HBAR_J_S = 1.054571817e-34
EV_J = 1.602176634e-19

DEFAULT_ETA_VALUES: tuple[float, ...] = (1e-8, 1e-7, 1e-6, 1e-5, 1e-4, 1e-3)  # workflows/ifc_bulk.py:54


def qe_omega_to_rad_s(omega):
    """QE-q2r internal omega -> rad/s (negfpy modeling/units.py:18-26)."""
    return np.asarray(omega) * np.sqrt(RYDBERG_J / (QE_RY_MASS_UNIT_KG * BOHR_M * BOHR_M))


def qe_omega_to_cm1(omega):
    """QE-q2r internal omega -> cm^-1 (negfpy modeling/units.py:36-40)."""
    return np.asarray(qe_omega_to_rad_s(omega), dtype=float) / (2.0 * np.pi * SPEED_OF_LIGHT_CM_S)


def qe_ev_to_omega(ev):
    """Phonon energy in eV -> QE-q2r internal omega (negfpy modeling/units.py:43-54)."""
    factor = float(np.asarray(qe_omega_to_rad_s(1.0), dtype=float)) * HBAR_J_S / EV_J
    return np.asarray(ev, dtype=float) / factor


def resolve_eta_values_for_omega(omega: float, omega_cm1: float, *, eta_values: tuple[float, ...],
                                 max_eta_over_omega: float | None, eta_ratio_cm1_min: float | None) -> tuple:
    """negfpy ``workflows/ifc_bulk.py:581-595``."""
    if max_eta_over_omega is None:
        return eta_values
    apply_cap = eta_ratio_cm1_min is None or omega_cm1 >= eta_ratio_cm1_min
    if not apply_cap:
        return eta_values
    filtered = tuple(e for e in eta_values if (e / omega) <= max_eta_over_omega)
    return filtered if len(filtered) > 0 else (min(eta_values),)


def resolve_parallel_solver_config(scfg: dict[str, Any]) -> dict[str, Any]:
    """negfpy ``workflows/ifc_bulk.py:598-617`` (reported, not used for execution)."""
    pcfg = dict(scfg.get("parallel", {}))
    enabled = bool(pcfg.get("enabled", False))
    backend = str(pcfg.get("backend", "thread")).lower()
    if backend not in {"thread", "process"}:
        raise ValueError("solver.parallel.backend must be one of: thread, process.")
    workers_raw = pcfg.get("workers", None)
    workers = int(os.cpu_count() or 1) if workers_raw is None else int(workers_raw)
    workers = max(workers, 1)
    blas_threads_raw = pcfg.get("blas_threads", 1 if enabled else None)
    blas_threads = None if blas_threads_raw is None else max(int(blas_threads_raw), 1)
    return {"enabled": enabled and workers > 1, "backend": backend, "workers": workers, "blas_threads": blas_threads}


class _Mesh:
    """The device-resident blocks of one k mesh, and the per-k acceptance limits."""

    def __init__(self, kpoints, device, lead_left, lead_right, eta_device, vdl_left, vdl_right, omega_scale,
                 max_channel_factor):
        self.kpoints = list(kpoints)
        fast = _material_fast_path(device, lead_left, lead_right, vdl_left, vdl_right, None, None, omega_scale)
        if fast is not None and self.kpoints:
            # All k blocks on the GPU; one k through the host path for the
            # validation, the omega scale and the device-eta rule.
            from .kspace import interface_system, stacked_system

            systems = _prepare_ladder_systems(1.0, device, lead_left, lead_right, self.kpoints[:1], eta_device,
                                              vdl_left, vdl_right, None, None, omega_scale)
            build = interface_system if fast[0] == "interface" else stacked_system
            self.sys = build(fast[1], fast[2], [() if k is None else k for k in self.kpoints])
        else:
            systems = _prepare_ladder_systems(1.0, device, lead_left, lead_right, self.kpoints, eta_device, vdl_left,
                                              vdl_right, None, None, omega_scale)
            self.sys, _ = stack_systems(systems)
        self.scale = systems[0]["scale"]
        self.eta_dev_for = systems[0]["_eta_dev_for"]
        nl = int(self.sys.nl)
        self.max_allowed = None if max_channel_factor is None else float(max_channel_factor) * float(nl)


def _solve(mesh: _Mesh, omegas: list, etas: list, ks: list) -> tuple[np.ndarray, np.ndarray]:
    """T and status of (omega, eta, k) points of one mesh in one launch."""
    dev = _lib.require_cuda()
    P = len(omegas)
    if P == 0:
        return np.zeros(0), np.zeros(0, dtype=np.int32)
    eds = [mesh.eta_dev_for(e) for e in etas]
    T = np.full(P, np.nan)
    st = np.full(P, -1, dtype=np.int32)
    ok = [i for i in range(P) if eds[i] >= 0.0]  # a negative device eta is negfpy's ValueError
    if ok:
        om = torch.tensor([omegas[i] / mesh.scale for i in ok], dtype=torch.float64, device=dev)
        et = torch.tensor([etas[i] / mesh.scale for i in ok], dtype=torch.float64, device=dev)
        ed = torch.tensor([eds[i] for i in ok], dtype=torch.float64, device=dev)
        ki = torch.tensor([ks[i] for i in ok], dtype=torch.int32, device=dev)
        r = mesh.sys.transmission(om, ki, et, ed)
        T[ok] = r["T"].cpu().numpy()
        st[ok] = r["status"].cpu().numpy()
    return T, st


def _rejected(omega, kp, eta, t, reason):
    return {"omega": float(omega), "kpar": tuple(float(x) for x in kp) if kp is not None else (), "eta": float(eta),
            "t": None if reason == "exception" else float(t), "reason": reason}


def run_transmission(cfg: dict[str, Any], *, device, lead_left, lead_right, device_to_lead_left=None,
                     device_to_lead_right=None, omegas: np.ndarray, kmesh: dict[str, Any]) -> dict[str, Any]:
    """k-averaged T(omega) of the workflow with its eta scheme, batched on the GPU.

    Same arguments, configuration keys and result dictionary as negfpy's
    ``_run_transmission`` (``workflows/ifc_bulk.py:1059-1288``)."""
    scfg = dict(cfg.get("solver", {}))
    sgf_method = str(scfg.get("surface_gf_method", "generalized_eigen_svd"))
    eta_scheme = str(scfg.get("eta_scheme", "adaptive")).lower().replace("-", "_")
    eta_fixed = float(scfg.get("eta_fixed", 1e-4))
    eta_values_base = tuple(float(v) for v in scfg.get("eta_values", DEFAULT_ETA_VALUES))
    eta_device_raw = scfg.get("eta_device", None)
    eta_device = None if eta_device_raw is None else float(eta_device_raw)
    min_success_fraction = float(scfg.get("min_success_fraction", 0.7))
    nonnegative_tolerance = float(scfg.get("nonnegative_tolerance", 1e-8))
    max_channel_factor_raw = scfg.get("max_channel_factor", 1.5)
    max_channel_factor = None if max_channel_factor_raw is None else float(max_channel_factor_raw)
    collect_rejected = bool(scfg.get("collect_rejected", False))
    max_eta_over_omega_raw = scfg.get("max_eta_over_omega", None)
    max_eta_over_omega = None if max_eta_over_omega_raw is None else float(max_eta_over_omega_raw)
    eta_ratio_cm1_min_raw = scfg.get("eta_ratio_cm1_min", None)
    eta_ratio_cm1_min = None if eta_ratio_cm1_min_raw is None else float(eta_ratio_cm1_min_raw)
    parallel_cfg = resolve_parallel_solver_config(scfg)
    omega_scale_mode = str(scfg.get("omega_scale_mode", "none")).lower()
    if omega_scale_mode == "ev":
        omega_scale = float(np.asarray(qe_ev_to_omega(1.0), dtype=float))
    elif omega_scale_mode == "none":
        omega_scale = None
    else:
        raise ValueError("solver.omega_scale_mode must be 'none' or 'ev'.")
    check_method(sgf_method)
    per_k = eta_scheme not in ("fixed", "adaptive_global")

    omegas = np.asarray(omegas, dtype=float)
    W = omegas.size
    vals = np.zeros(W, dtype=float)
    results: list[dict | None] = [None] * W
    meshes: dict[str, _Mesh] = {}
    tasks = []  # (index, omega, omega_cm1, mesh name, eta ladder)
    for i, w in enumerate(omegas):
        w = float(w)
        if w <= 0.0:
            results[i] = {"value": 0.0, "eta_record": None, "failure": None}
            continue
        w_cm1 = float(np.asarray(qe_omega_to_cm1(w), dtype=float))
        use_low = bool(w_cm1 <= float(kmesh["low_cm1"]))
        name = "low" if use_low else "high"
        ladder = resolve_eta_values_for_omega(w, w_cm1, eta_values=eta_values_base,
                                              max_eta_over_omega=max_eta_over_omega,
                                              eta_ratio_cm1_min=eta_ratio_cm1_min)
        if eta_scheme == "fixed":
            ladder = (eta_fixed,)
        kpts = kmesh[name]["kpoints"]
        try:
            _check_adaptive_args(kpts, ladder, min_success_fraction, nonnegative_tolerance, max_channel_factor)
        except Exception as exc:  # negfpy's task turns every exception into a failure record
            results[i] = {"value": np.nan, "eta_record": None,
                          "failure": {"omega_qe": w, "omega_cm1": w_cm1, "error": str(exc)}}
            continue
        if name not in meshes:
            meshes[name] = _Mesh(kpts, device, lead_left, lead_right, eta_device, device_to_lead_left,
                                 device_to_lead_right, omega_scale, max_channel_factor)
        tasks.append((i, w, w_cm1, name, tuple(float(e) for e in ladder)))

    # ladder state
    state = {}
    for i, w, w_cm1, name, ladder in tasks:
        K = len(meshes[name].kpoints)
        state[i] = {"pending": list(range(K)), "accepted": {}, "attempts": [], "done": False, "rej_all": [],
                    "K": K, "name": name, "w": w, "ladder": ladder}
    rung = 0
    while True:
        batch: dict[str, list] = {}
        for i, w, w_cm1, name, ladder in tasks:
            s = state[i]
            if s["done"] or rung >= len(ladder) or not s["pending"]:
                continue
            for ki in s["pending"]:
                batch.setdefault(name, []).append((i, ki, ladder[rung]))
        if not batch:
            break
        for name, pts in batch.items():
            mesh = meshes[name]
            T, st = _solve(mesh, [state[i]["w"] for i, _, _ in pts], [e for _, _, e in pts], [k for _, k, _ in pts])
            outcome: dict[int, list] = {}
            for (i, ki, eta), t, sv in zip(pts, T, st):
                outcome.setdefault(i, []).append((ki, eta, t, sv))
            for i, rows in outcome.items():
                s = state[i]
                kpts = mesh.kpoints
                if per_k:
                    nxt = []
                    for ki, eta, t, sv in rows:
                        reason = _classify(t, sv, mesh.max_allowed, nonnegative_tolerance)
                        if reason is None:
                            s["accepted"][ki] = (float(max(t, 0.0)), float(eta))
                        else:
                            s["attempts"].append((ki, rung, _rejected(s["w"], kpts[ki], eta, t, reason)))
                            nxt.append(ki)
                    s["pending"] = nxt
                else:
                    good = []
                    for ki, eta, t, sv in rows:
                        reason = _classify(t, sv, mesh.max_allowed, nonnegative_tolerance)
                        if reason is None:
                            good.append(float(max(t, 0.0)))
                        elif collect_rejected:
                            s["rej_all"].append(_rejected(s["w"], kpts[ki], eta, t, reason))
                    frac = float(len(good) / s["K"])
                    if good and frac >= min_success_fraction:
                        eta = rows[0][1]
                        s["done"] = True
                        s["value"] = float(np.mean(good))
                        s["info"] = {"n_total": s["K"], "n_success": len(good), "n_failed": s["K"] - len(good),
                                     "success_fraction": frac, "eta_selected": float(eta),
                                     "eta_histogram": {float(e): (len(good) if float(e) == float(eta) else 0)
                                                       for e in s["ladder"]}}
                        if collect_rejected:
                            s["info"]["n_rejected"] = len(s["rej_all"])
                            s["info"]["rejected"] = s["rej_all"]
        rung += 1

    for i, w, w_cm1, name, ladder in tasks:
        s = state[i]
        try:
            if per_k:
                K = s["K"]
                acc = s["accepted"]
                v = [acc[k][0] for k in range(K) if k in acc]
                used = [acc[k][1] for k in range(K) if k in acc]
                frac = float(len(v) / K)
                if not v:
                    raise RuntimeError("No k-point converged for adaptive k-averaged transmission.")
                if frac < min_success_fraction:
                    raise RuntimeError("Adaptive k-averaged transmission failed success-fraction threshold "
                                       f"(got {frac:.3f}, required >= {min_success_fraction:.3f}).")
                info = {"n_total": K, "n_success": len(v), "n_failed": K - len(v), "success_fraction": frac,
                        "eta_histogram": {float(e): int(sum(1 for u in used if u == float(e))) for e in ladder}}
                if collect_rejected:
                    rej = [a[2] for a in sorted(s["attempts"], key=lambda a: (a[0], a[1]))]
                    info["n_rejected"] = len(rej)
                    info["rejected"] = rej
                tval = float(np.mean(v))
            else:
                if not s["done"]:
                    raise RuntimeError("No eta value satisfied global adaptive k-averaging quality threshold "
                                       f"(required success_fraction >= {min_success_fraction:.3f}).")
                info, tval = s["info"], s["value"]
        except Exception as exc:
            results[i] = {"value": np.nan, "eta_record": None,
                          "failure": {"omega_qe": w, "omega_cm1": w_cm1, "error": str(exc)}}
            continue
        hist = dict(info.get("eta_histogram", {}))
        used_e = [float(e) for e, c in hist.items() if int(c) > 0]
        max_eta_used = max(used_e) if used_e else np.nan
        results[i] = {
            "value": tval,
            "eta_record": {
                "omega_qe": w, "omega_cm1": w_cm1, "n_failed_kpoints": int(info.get("n_failed", 0)),
                "success_fraction": float(info.get("success_fraction", 0.0)), "eta_histogram": hist,
                "eta_selected": info.get("eta_selected", None),
                "max_eta_used": None if not np.isfinite(max_eta_used) else float(max_eta_used),
                "max_eta_over_omega": None if not np.isfinite(max_eta_used) else float(max_eta_used / w),
            },
            "failure": None,
            "n_rejected": int(info.get("n_rejected", 0)) if collect_rejected else 0,
        }

    rejected_total = 0
    for i, r in enumerate(results):
        vals[i] = float(r["value"])
        if r["failure"] is None and collect_rejected:
            rejected_total += int(r.get("n_rejected", 0))
    eta_records = [r["eta_record"] for r in results if r["eta_record"] is not None]
    omega_failures = [r["failure"] for r in results if r["failure"] is not None]
    if np.all(~np.isfinite(vals)):
        raise RuntimeError("Transmission calculation failed for all omega points.")
    vals = np.where(np.isfinite(vals), vals, np.nan)
    vals = np.where(vals < 0.0, np.maximum(vals, -1e-12), vals)
    vals = np.where(np.isfinite(vals), np.clip(vals, 0.0, None), np.nan)
    max_ratio = max((r["max_eta_over_omega"] for r in eta_records if r["max_eta_over_omega"] is not None),
                    default=None)
    return {
        "values": vals,
        "eta_records": eta_records,
        "omega_failures": omega_failures,
        "n_rejected_total": int(rejected_total),
        "summary": {
            "surface_gf_method": sgf_method,
            "eta_scheme": eta_scheme,
            "eta_fixed": eta_fixed,
            "eta_values_base": eta_values_base,
            "eta_device": eta_device,
            "parallel": {"enabled": bool(parallel_cfg["enabled"]), "backend": str(parallel_cfg["backend"]),
                         "workers": int(parallel_cfg["workers"]), "blas_threads": parallel_cfg["blas_threads"]},
            "max_eta_over_omega": max_ratio,
            "n_omega_failures": len(omega_failures),
        },
    }


def compute_fcs_k_moments(cfg: dict[str, Any], *, device, lead_left, lead_right, device_to_lead_left=None,
                          device_to_lead_right=None, omegas: np.ndarray, kmesh: dict[str, Any]) -> dict[str, Any]:
    """<T>_k and <T^2>_k per omega with one eta per omega (negfpy
    ``workflows/ifc_bulk.py:1690-1784``, ``_compute_fcs_k_moments``).

    The first eta of the omega's ladder (or ``eta_fixed``) at which at least
    one k point and at least ``min_success_fraction`` of them give a finite T
    no lower than ``-nonnegative_tolerance`` is taken; the moments are the
    means of max(T, 0) and its square over those k points.  Each rung is ONE
    launch per k mesh over every omega still without an accepted eta."""
    scfg = dict(cfg.get("solver", {}))
    sgf_method = str(scfg.get("surface_gf_method", "generalized_eigen_svd"))
    eta_fixed = float(scfg.get("eta_fixed", 1e-4))
    eta_values_base = tuple(float(v) for v in scfg.get("eta_values", DEFAULT_ETA_VALUES))
    eta_device_raw = scfg.get("eta_device", None)
    eta_device = None if eta_device_raw is None else float(eta_device_raw)
    min_success_fraction = float(scfg.get("min_success_fraction", 0.7))
    nonnegative_tolerance = float(scfg.get("nonnegative_tolerance", 1e-8))
    max_eta_over_omega_raw = scfg.get("max_eta_over_omega", None)
    max_eta_over_omega = None if max_eta_over_omega_raw is None else float(max_eta_over_omega_raw)
    eta_ratio_cm1_min_raw = scfg.get("eta_ratio_cm1_min", None)
    eta_ratio_cm1_min = None if eta_ratio_cm1_min_raw is None else float(eta_ratio_cm1_min_raw)
    eta_scheme = str(scfg.get("eta_scheme", "adaptive_global")).lower().replace("-", "_")
    if eta_scheme not in {"fixed", "adaptive_global"}:
        eta_scheme = "adaptive_global"
    check_method(sgf_method)

    omegas = np.asarray(omegas, dtype=float)
    W = int(omegas.size)
    t_mean = np.full((W,), np.nan, dtype=float)
    t2_mean = np.full((W,), np.nan, dtype=float)
    eta_selected = np.full((W,), np.nan, dtype=float)
    n_k_success = np.zeros((W,), dtype=int)
    meshes: dict[str, _Mesh] = {}
    tasks = {}  # omega index -> [omega, omega_cm1, mesh name, etas to try]
    for i, w in enumerate(omegas):
        w = float(w)
        if w <= 0.0:
            t_mean[i] = 0.0
            t2_mean[i] = 0.0
            continue
        w_cm1 = float(np.asarray(qe_omega_to_cm1(w), dtype=float))
        name = "low" if w_cm1 <= float(kmesh["low_cm1"]) else "high"
        ladder = resolve_eta_values_for_omega(w, w_cm1, eta_values=eta_values_base,
                                              max_eta_over_omega=max_eta_over_omega,
                                              eta_ratio_cm1_min=eta_ratio_cm1_min)
        eta_try = (eta_fixed,) if eta_scheme == "fixed" else ladder
        if len(kmesh[name]["kpoints"]) > 0 and name not in meshes:
            meshes[name] = _Mesh(kmesh[name]["kpoints"], device, lead_left, lead_right, eta_device,
                                 device_to_lead_left, device_to_lead_right, None, None)
        tasks[i] = [w, w_cm1, name, tuple(float(e) for e in eta_try)]

    pending = [i for i in tasks if tasks[i][2] in meshes]
    rung = 0
    while pending:
        batch: dict[str, list] = {}
        for i in pending:
            w, _, name, etas = tasks[i]
            if rung < len(etas):
                batch.setdefault(name, []).extend((i, k) for k in range(len(meshes[name].kpoints)))
        if not batch:
            break
        done = set()
        for name, pts in batch.items():
            mesh = meshes[name]
            K = len(mesh.kpoints)
            T, st = _solve(mesh, [tasks[i][0] for i, _ in pts], [tasks[i][3][rung] for i, _ in pts],
                           [k for _, k in pts])
            for j in range(0, len(pts), K):
                i = pts[j][0]
                vals = np.array([max(float(t), 0.0) for t, s in zip(T[j:j + K], st[j:j + K])
                                 if _classify(t, s, None, nonnegative_tolerance) is None], dtype=float)
                frac = float(vals.size / max(K, 1))
                if vals.size > 0 and frac >= min_success_fraction:
                    t_mean[i] = float(np.mean(vals))
                    t2_mean[i] = float(np.mean(vals * vals))
                    eta_selected[i] = tasks[i][3][rung]
                    n_k_success[i] = int(vals.size)
                    done.add(i)
        pending = [i for i in pending if i not in done]
        rung += 1
    omega_failures = [{"omega_qe": tasks[i][0], "omega_cm1": tasks[i][1], "reason": "no_eta_passed_threshold"}
                      for i in sorted(tasks) if not np.isfinite(t_mean[i])]
    return {"t_mean": t_mean, "t2_mean": t2_mean, "eta_selected": eta_selected, "n_k_success": n_k_success,
            "omega_failures": omega_failures}


def run_fcs(cfg: dict[str, Any], *, omegas: np.ndarray, kmesh: dict[str, Any], device, lead_left, lead_right,
            device_to_lead_left=None, device_to_lead_right=None, area_m2: float | None) -> dict[str, Any]:
    """The workflow's full-counting-statistics stage (negfpy
    ``workflows/ifc_bulk.py:1787-1935``, ``_run_fcs``): the k moments
    (``compute_fcs_k_moments``), then C1, C2 and the finite-time uncertainty
    over the temperature sweep, with the spectral integrals on the GPU.  Same
    configuration keys, checks, messages and result dictionary."""
    from .fcs import heat_current_cumulants_from_k_moments, heat_current_uncertainty

    fcfg = dict(cfg.get("fcs", {}))
    x_mode = str(fcfg.get("x", "temperature")).lower().replace("-", "_")
    y_mode = str(fcfg.get("y", "conductance_per_area")).lower().replace("-", "_")
    if x_mode not in {"temperature", "temperature_bias"}:
        raise ValueError("fcs.x must be 'temperature' or 'temperature_bias'.")
    if y_mode not in {"heat_current", "heat_current_per_area", "conductance", "conductance_per_area"}:
        raise ValueError("fcs.y must be one of: heat_current, heat_current_per_area, conductance, conductance_per_area.")
    t_min = float(fcfg.get("temperature_min_k", 50.0))
    t_max = float(fcfg.get("temperature_max_k", 1000.0))
    n_points = int(fcfg.get("n_points", 120))
    tau_s = float(fcfg.get("measurement_time_s", 1e-6))
    if n_points < 2:
        raise ValueError("fcs.n_points must be >= 2.")
    if tau_s <= 0.0:
        raise ValueError("fcs.measurement_time_s must be positive.")

    moments = compute_fcs_k_moments(cfg, device=device, lead_left=lead_left, lead_right=lead_right,
                                    device_to_lead_left=device_to_lead_left, device_to_lead_right=device_to_lead_right,
                                    omegas=omegas, kmesh=kmesh)
    omega_rad_s = np.asarray(qe_omega_to_rad_s(omegas), dtype=float)
    valid = np.isfinite(moments["t_mean"]) & np.isfinite(moments["t2_mean"])
    if int(np.sum(valid)) < 2:
        raise RuntimeError("FCS failed: insufficient converged omega points.")
    om = omega_rad_s[valid]
    t1 = np.asarray(moments["t_mean"], dtype=float)[valid]
    t2 = np.asarray(moments["t2_mean"], dtype=float)[valid]

    xvals = np.linspace(t_min, t_max, n_points, endpoint=True)
    if x_mode == "temperature":
        temp_mode = str(fcfg.get("temperature_mode", "fixed_delta")).lower().replace("-", "_")
        if temp_mode == "fixed_right":
            t_left = xvals
            t_right = np.full_like(xvals, float(fcfg.get("temperature_right_k", 300.0)))
            x_label = "Temperature Left (K)"
        else:
            dT = float(fcfg.get("delta_t_k", 10.0))
            if dT <= 0.0:
                raise ValueError("fcs.delta_t_k must be positive.")
            t_left = xvals + 0.5 * dT
            t_right = xvals - 0.5 * dT
            x_label = "Average Temperature (K)"
    else:
        tavg = float(fcfg.get("temperature_avg_k", 300.0))
        t_left = tavg + 0.5 * xvals
        t_right = tavg - 0.5 * xvals
        x_label = "Temperature Bias (K)"
    if np.any(t_left <= 0.0) or np.any(t_right <= 0.0):
        raise ValueError("FCS sweep generates non-positive temperatures.")

    y = np.zeros_like(xvals, dtype=float)
    y_std = np.zeros_like(xvals, dtype=float)
    c1 = np.zeros_like(xvals, dtype=float)
    c2 = np.zeros_like(xvals, dtype=float)
    for i in range(xvals.size):
        cc = heat_current_cumulants_from_k_moments(om, t1, t2, float(t_left[i]), float(t_right[i]))
        uu = heat_current_uncertainty(cc, measurement_time_s=tau_s)
        c1[i] = float(cc.c1_j_per_s)
        c2[i] = float(cc.c2_j2_per_s)
        if y_mode in {"conductance", "conductance_per_area"}:
            dtemp = float(t_left[i] - t_right[i])
            if abs(dtemp) < 1e-12:
                y[i] = np.nan
                y_std[i] = np.nan
            else:
                y[i] = float(c1[i] / dtemp)
                y_std[i] = float(uu.std_current_j_per_s / abs(dtemp))
        else:
            y[i] = float(c1[i])
            y_std[i] = float(uu.std_current_j_per_s)
    if y_mode in {"heat_current_per_area", "conductance_per_area"}:
        if area_m2 is None or area_m2 <= 0.0:
            raise ValueError("FCS y-mode requests per-area quantity but area is unavailable.")
        y = y / float(area_m2)
        y_std = y_std / float(area_m2)
    y_label = {"heat_current": "Heat Current (J/s)", "heat_current_per_area": "Heat Current per Area (J/s/m^2)",
               "conductance": "Thermal Conductance (W/K)"}.get(y_mode, "Thermal Conductance per Area (W/m^2/K)")
    n_conv = int(np.sum(valid))
    return {
        "x_mode": x_mode, "x_label": x_label, "y_mode": y_mode, "y_label": y_label, "x": xvals,
        "temp_left_k": t_left, "temp_right_k": t_right, "y": y, "y_std": y_std, "c1_j_per_s": c1,
        "c2_j2_per_s": c2, "measurement_time_s": float(tau_s), "omega_qe": np.asarray(omegas, dtype=float),
        "omega_rad_s_valid": om, "t_mean_valid": t1, "t2_mean_valid": t2,
        "t_mean": np.asarray(moments["t_mean"], dtype=float), "t2_mean": np.asarray(moments["t2_mean"], dtype=float),
        "eta_selected": np.asarray(moments["eta_selected"], dtype=float),
        "n_k_success": np.asarray(moments["n_k_success"], dtype=int),
        "omega_failures": list(moments["omega_failures"]), "n_omega_converged": n_conv,
        "n_omega_total": int(len(omegas)),
        "summary": {"x_mode": x_mode, "y_mode": y_mode, "measurement_time_s": float(tau_s),
                    "n_omega_converged": n_conv, "n_omega_total": int(len(omegas))},
    }


class _DosMesh:
    """One k mesh of a lead, stacked once on the GPU for the DOS stage."""

    def __init__(self, lead, kpoints):
        from .dos import _stack_leads
        from . import engine

        self.kpoints = list(kpoints)
        self.K = len(self.kpoints)
        if self.K:
            d00, d01, d10 = _stack_leads(lead, [k if len(k) > 0 else None for k in self.kpoints])
            self.n = int(d00.shape[-1])
            self.blocks = (engine._c(d00), engine._c(d01), None if d10 is None else engine._c(d10))

    def solve(self, omegas: list, etas: list, ks: list, normalize_per_mode: bool):
        """DOS and status of (omega, eta, k) points in one launch."""
        from . import engine

        dev = _lib.require_cuda()
        if not omegas:
            return np.zeros(0), np.zeros(0, dtype=np.int32)
        r = engine.sgf_sr(*self.blocks, torch.tensor(omegas, dtype=torch.float64, device=dev),
                          torch.tensor(etas, dtype=torch.float64, device=dev),
                          torch.tensor(ks, dtype=torch.int32, device=dev), want_g=False, want_dos=True)
        d = r["dos"].cpu().numpy()
        return (d / self.n if normalize_per_mode else d), r["status"].cpu().numpy()


def run_dos(cfg: dict[str, Any], *, lead, omegas: np.ndarray, kmesh: dict[str, Any]) -> dict[str, Any]:
    """The workflow's surface-DOS stage (negfpy ``workflows/ifc_bulk.py:1290-1441``,
    ``_run_dos``, with ``_lead_surface_dos_kavg_adaptive_global_eta``
    ``:908-948``): per omega the k-mean DOS at ``eta_fixed``, with one eta per
    omega (``adaptive_global``), or with negfpy's per-k ladder (any other
    scheme), batched: each rung is ONE launch per k mesh over all pending
    (omega, k) points.  Same configuration keys, acceptance rules, messages
    and result dictionary."""
    from .surface_gf import raise_for_status

    scfg = dict(cfg.get("solver", {}))
    dcfg = dict(cfg.get("dos", {}))
    sgf_method = str(scfg.get("surface_gf_method", "generalized_eigen_svd"))
    eta_scheme = str(scfg.get("eta_scheme", "adaptive")).lower().replace("-", "_")
    eta_fixed = float(scfg.get("eta_fixed", 1e-4))
    eta_values_base = tuple(float(v) for v in scfg.get("eta_values", DEFAULT_ETA_VALUES))
    min_success_fraction = float(scfg.get("min_success_fraction", 0.7))
    max_eta_over_omega_raw = scfg.get("max_eta_over_omega", None)
    max_eta_over_omega = None if max_eta_over_omega_raw is None else float(max_eta_over_omega_raw)
    eta_ratio_cm1_min_raw = scfg.get("eta_ratio_cm1_min", None)
    eta_ratio_cm1_min = None if eta_ratio_cm1_min_raw is None else float(eta_ratio_cm1_min_raw)
    normalize_per_mode = bool(dcfg.get("normalize_per_mode", False))
    negative_tolerance = float(dcfg.get("negative_tolerance", 1e-12))
    check_method(sgf_method)

    omegas = np.asarray(omegas, dtype=float)
    vals = np.zeros_like(omegas, dtype=float)
    meshes: dict[str, _DosMesh] = {}
    tasks: dict[int, dict] = {}
    outcome: dict[int, tuple] = {}  # omega index -> (dos, info) or (None, error message)
    for i, w in enumerate(omegas):
        w = float(w)
        if w < 0.0:
            vals[i] = np.nan
            continue
        w_cm1 = float(np.asarray(qe_omega_to_cm1(w), dtype=float))
        name = "low" if w_cm1 <= float(kmesh["low_cm1"]) else "high"
        ladder = resolve_eta_values_for_omega(float(max(w, 1e-30)), w_cm1, eta_values=eta_values_base,
                                              max_eta_over_omega=max_eta_over_omega,
                                              eta_ratio_cm1_min=eta_ratio_cm1_min)
        if name not in meshes:
            meshes[name] = _DosMesh(lead, kmesh[name]["kpoints"])
        K = meshes[name].K
        t = {"w": w, "w_cm1": w_cm1, "name": name, "K": K}
        if eta_scheme == "fixed":
            if K == 0:
                outcome[i] = (None, "kpoints must contain at least one k-point.")
                continue
            t["etas"], t["rule"] = (eta_fixed,), "fixed"
        elif eta_scheme == "adaptive_global":
            if K == 0 and ladder:
                outcome[i] = (None, "division by zero")
                continue
            t["etas"], t["rule"] = ladder, "global"
        else:
            if K == 0:
                outcome[i] = (None, "kpoints must contain at least one k-point.")
                continue
            if len(ladder) == 0:
                outcome[i] = (None, "eta_values must contain at least one eta value.")
                continue
            if not (0.0 <= min_success_fraction <= 1.0):
                outcome[i] = (None, "min_success_fraction must be in [0, 1].")
                continue
            t["etas"], t["rule"] = ladder, "per_k"
            t["pending"], t["accepted"] = list(range(K)), {}
        tasks[i] = t

    pending = list(tasks)
    rung = 0
    while pending:
        batch: dict[str, list] = {}
        for i in pending:
            t = tasks[i]
            if rung < len(t["etas"]):
                ks = t["pending"] if t["rule"] == "per_k" else range(t["K"])
                batch.setdefault(t["name"], []).extend((i, k) for k in ks)
        if not batch:
            break
        done = set()
        for name, pts in batch.items():
            d, st = meshes[name].solve([tasks[i]["w"] for i, _ in pts], [tasks[i]["etas"][rung] for i, _ in pts],
                                       [k for _, k in pts], normalize_per_mode)
            rows: dict[int, list] = {}
            for (i, k), dv, sv in zip(pts, d, st):
                rows.setdefault(i, []).append((k, float(dv), int(sv)))
            for i, rr in rows.items():
                t = tasks[i]
                eta = t["etas"][rung]
                if t["rule"] == "fixed":
                    bad = [sv for _, _, sv in rr if sv != _lib.OK]
                    if bad:
                        try:
                            raise_for_status(bad[0])
                        except Exception as exc:  # negfpy's first failing k ends the k mean
                            outcome[i] = (None, str(exc))
                    else:
                        K = t["K"]
                        outcome[i] = (float(np.mean([dv for _, dv, _ in rr])),
                                      {"n_total": K, "n_success": K, "n_failed": 0, "success_fraction": 1.0,
                                       "eta_selected": float(eta_fixed), "eta_histogram": {float(eta_fixed): K}})
                    done.add(i)
                elif t["rule"] == "global":
                    good = [float(max(dv, 0.0)) for _, dv, sv in rr
                            if sv == _lib.OK and np.isfinite(dv) and not dv < -negative_tolerance]
                    frac = float(len(good) / t["K"])
                    if good and frac >= min_success_fraction:
                        outcome[i] = (float(np.mean(good)),
                                      {"n_total": t["K"], "n_success": len(good), "n_failed": t["K"] - len(good),
                                       "success_fraction": frac, "eta_selected": float(eta),
                                       "eta_histogram": {float(e): (len(good) if float(e) == float(eta) else 0)
                                                         for e in t["etas"]}})
                        done.add(i)
                else:
                    nxt = []
                    for k, dv, sv in rr:
                        if sv == _lib.OK and np.isfinite(dv):
                            t["accepted"][k] = (dv, float(eta))
                        else:
                            nxt.append(k)
                    t["pending"] = nxt
                    if not nxt:
                        done.add(i)
        pending = [i for i in pending if i not in done]
        rung += 1

    for i, t in tasks.items():
        if i in outcome:
            continue
        if t["rule"] == "global":
            outcome[i] = (None, "No eta value satisfied global adaptive DOS quality threshold.")
            continue
        K, acc = t["K"], t["accepted"]
        v = [acc[k][0] for k in range(K) if k in acc]
        used = [acc[k][1] for k in range(K) if k in acc]
        frac = float(len(v) / K)
        if not v:
            outcome[i] = (None, "No k-point converged for adaptive k-averaged DOS.")
        elif frac < min_success_fraction:
            outcome[i] = (None, "Adaptive k-averaged DOS failed success-fraction threshold "
                                f"(got {frac:.3f}, required >= {min_success_fraction:.3f}).")
        else:
            outcome[i] = (float(np.mean(v)), {"n_total": K, "n_success": len(v), "n_failed": K - len(v),
                                              "success_fraction": frac,
                                              "eta_histogram": {float(e): int(sum(1 for u in used if u == float(e)))
                                                                for e in t["etas"]}})

    eta_records, omega_failures = [], []
    for i in sorted(outcome):
        w = float(omegas[i])
        w_cm1 = float(np.asarray(qe_omega_to_cm1(w), dtype=float))
        dval, info = outcome[i]
        if dval is None:
            vals[i] = np.nan
            omega_failures.append({"omega_qe": w, "omega_cm1": w_cm1, "error": info})
            continue
        vals[i] = float(max(dval, 0.0))
        hist = dict(info.get("eta_histogram", {}))
        used_e = [float(e) for e, c in hist.items() if int(c) > 0]
        max_eta_used = max(used_e) if used_e else np.nan
        eta_records.append({
            "omega_qe": w, "omega_cm1": w_cm1, "n_failed_kpoints": int(info.get("n_failed", 0)),
            "success_fraction": float(info.get("success_fraction", 0.0)), "eta_histogram": hist,
            "eta_selected": info.get("eta_selected", None),
            "max_eta_used": None if not np.isfinite(max_eta_used) else float(max_eta_used),
            "max_eta_over_omega": None if not np.isfinite(max_eta_used) or w <= 0.0 else float(max_eta_used / w),
        })
    if np.all(~np.isfinite(vals)):
        raise RuntimeError("DOS calculation failed for all omega points.")
    max_ratio = max((r["max_eta_over_omega"] for r in eta_records if r["max_eta_over_omega"] is not None),
                    default=None)
    return {
        "values": vals,
        "eta_records": eta_records,
        "omega_failures": omega_failures,
        "summary": {"surface_gf_method": sgf_method, "eta_scheme": eta_scheme, "eta_fixed": eta_fixed,
                    "eta_values_base": eta_values_base, "normalize_per_mode": normalize_per_mode,
                    "max_eta_over_omega": max_ratio, "n_omega_failures": len(omega_failures)},
    }
