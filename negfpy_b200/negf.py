"""Drop-in transmission API (negfpy ``core/negf.py``) on the batched GPU engine.

Host side of each call: resolve the k-dependent blocks once per k, validate
arguments with negfpy's checks and messages, embed the contact couplings,
stack everything per k and upload.  Device side: one Sancho-Rubio launch per
distinct lead and one RGF launch for all points of the call.

The device solve is a recursive Green's function sweep, which needs the left
contact DOFs inside the first principal layer and the right contact DOFs
inside the last one.  negfpy's defaults (first n_cL / last n_cR DOFs, with
n_c equal to the lead block order) always satisfy this; other index sets
raise ``ValueError``.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib, engine
from .surface_gf import check_method, raise_for_status
from .types import resolve_device, resolve_lead_blocks

Array = np.ndarray


def _resolve_coupling(coupling, kpar):
    """negfpy ``negf.py:41-50``: array or callable of k."""
    if coupling is None:
        return None
    if callable(coupling):
        return np.asarray(coupling(kpar), dtype=np.complex128)
    return np.asarray(coupling, dtype=np.complex128)


def _normalize_contact_indices(indices, *, dim: int, default: Array) -> Array:
    """negfpy ``negf.py:119-138``."""
    if indices is None:
        idx = np.asarray(default, dtype=int).ravel()
    elif isinstance(indices, slice):
        idx = np.arange(dim, dtype=int)[indices]
    else:
        idx = np.asarray(indices, dtype=int).ravel()
    if idx.size == 0:
        raise ValueError("Contact indices must be non-empty.")
    if np.any(idx < 0) or np.any(idx >= dim):
        raise ValueError("Contact indices out of device range.")
    if np.unique(idx).size != idx.size:
        raise ValueError("Contact indices must be unique.")
    return idx


def _scaled(a, s2):
    return np.asarray(a, dtype=np.complex128) / s2


def point_system(omega, device, lead_left, lead_right, eta, eta_device=None, kpar=None, device_to_lead_left=None,
                 device_to_lead_right=None, contact_left_indices=None, contact_right_indices=None,
                 omega_scale=None) -> dict:
    """Resolved, validated and scaled inputs of one (omega, k) point.

    Follows negfpy ``negf.py:141-250`` step by step (eta_device check, the
    omega_scale rescale of omega/eta/blocks/couplings, default couplings and
    contacts, index checks, coupling shape checks) and returns host arrays:
    onsite ``[L, n, n]``, coupling ``[L-1, n, n]``, lead tuples, embedded
    couplings ``vl`` ``[n, nl]`` / ``vr`` ``[n, nr]`` and the effective
    omega / eta values.
    """
    dev = resolve_device(device, kpar)
    vdl_left = _resolve_coupling(device_to_lead_left, kpar)
    vdl_right = _resolve_coupling(device_to_lead_right, kpar)
    left = resolve_lead_blocks(lead_left, kpar)
    right = resolve_lead_blocks(lead_right, kpar)
    npl = dev.dof_per_layer
    L = dev.n_layers
    dim = L * npl
    eta_dev = float(eta if eta_device is None else eta_device)
    if eta_dev < 0.0:
        raise ValueError("eta_device must be non-negative.")
    eta_lead = float(eta)
    omega_eff = float(omega)
    onsite = [np.asarray(b, dtype=np.complex128) for b in dev.onsite_blocks]
    coupling = [np.asarray(b, dtype=np.complex128) for b in dev.coupling_blocks]
    ll = [np.asarray(left.d00, dtype=np.complex128), np.asarray(left.d01, dtype=np.complex128),
          None if left.d10 is None else np.asarray(left.d10, dtype=np.complex128)]
    lr = [np.asarray(right.d00, dtype=np.complex128), np.asarray(right.d01, dtype=np.complex128),
          None if right.d10 is None else np.asarray(right.d10, dtype=np.complex128)]
    if omega_scale is not None:
        scale = float(omega_scale)
        if scale <= 0.0:
            raise ValueError("omega_scale must be positive when provided.")
        s2 = scale * scale
        omega_eff /= scale
        eta_lead /= scale
        eta_dev /= scale
        onsite = [_scaled(b, s2) for b in onsite]
        coupling = [_scaled(b, s2) for b in coupling]
        ll = [None if b is None else _scaled(b, s2) for b in ll]
        lr = [None if b is None else _scaled(b, s2) for b in lr]
    if vdl_left is None:
        vdl_left = ll[2] if ll[2] is not None else ll[1].conj().T
    if vdl_right is None:
        vdl_right = lr[1]
    if omega_scale is not None:
        # negfpy divides every contact coupling by s^2 here, the defaults
        # included although they come from the already rescaled lead blocks
        # (core/negf.py:192-204); kept identical for parity.
        s2 = float(omega_scale) * float(omega_scale)
        vdl_left = vdl_left / s2
        vdl_right = vdl_right / s2
    ncl, ncr = vdl_left.shape[0], vdl_right.shape[0]
    idx_l = _normalize_contact_indices(contact_left_indices, dim=dim, default=np.arange(ncl, dtype=int))
    idx_r = _normalize_contact_indices(contact_right_indices, dim=dim, default=np.arange(dim - ncr, dim, dtype=int))
    if idx_l.size != ncl:
        raise ValueError(f"Left contact index count must match device_to_lead_left rows (got {idx_l.size}, expected {ncl}).")
    if idx_r.size != ncr:
        raise ValueError(f"Right contact index count must match device_to_lead_right rows (got {idx_r.size}, expected {ncr}).")
    for v, lead in ((vdl_left, ll), (vdl_right, lr)):
        if v.ndim != 2:
            raise ValueError("device_to_lead coupling must be a 2D array.")
        if v.shape[1] != lead[0].shape[0]:
            raise ValueError("device_to_lead coupling has incompatible lead dimension "
                             f"(got {v.shape[1]}, expected {lead[0].shape[0]}).")
    if np.any(idx_l >= npl):
        raise ValueError("Left contact indices must lie in the first principal layer for the RGF device solve.")
    loc_r = idx_r - (L - 1) * npl
    if np.any(loc_r < 0):
        raise ValueError("Right contact indices must lie in the last principal layer for the RGF device solve.")
    vl = np.zeros((npl, ll[0].shape[0]), dtype=np.complex128)
    vl[idx_l, :] = vdl_left
    vr = np.zeros((npl, lr[0].shape[0]), dtype=np.complex128)
    vr[loc_r, :] = vdl_right
    return {
        "onsite": np.stack(onsite),
        "coupling": np.stack(coupling) if L > 1 else np.zeros((1, npl, npl), dtype=np.complex128),
        "lead_l": ll, "lead_r": lr, "vl": vl, "vr": vr, "n_layers": L,
        "omega": omega_eff, "eta": eta_lead, "eta_dev": eta_dev,
    }


def _same_lead(a: list, b: list) -> bool:
    for x, y in zip(a, b):
        if (x is None) != (y is None):
            return False
        if x is not None and (x.shape != y.shape or not np.array_equal(x, y)):
            return False
    return True


def stack_systems(systems: list[dict]) -> tuple[engine.StackedSystem, dict]:
    """Stack per-k point systems into one device-resident ``StackedSystem``."""
    def lead(key):
        d10s = [s[key][2] for s in systems]
        return {"d00": np.stack([s[key][0] for s in systems]), "d01": np.stack([s[key][1] for s in systems]),
                "d10": None if any(d is None for d in d10s) else np.stack(d10s)}

    ll = lead("lead_l")
    same = all(_same_lead(s["lead_l"], s["lead_r"]) for s in systems)
    lr = ll if same else lead("lead_r")
    shapes = {(s["onsite"].shape, s["vl"].shape, s["vr"].shape, s["n_layers"]) for s in systems}
    if len(shapes) != 1:
        raise ValueError("all k-points of one call must share block shapes")
    onsite = np.stack([s["onsite"] for s in systems])
    coupling = np.stack([s["coupling"] for s in systems])
    # Identical layers are stored once (layer stride 0 in the kernel).
    uniform = bool(np.all(onsite == onsite[:, :1]) and np.all(coupling == coupling[:, :1]))
    if uniform:
        onsite, coupling = onsite[:, :1], coupling[:, :1]
    sysobj = engine.StackedSystem.from_arrays(
        ll, lr, onsite, coupling, systems[0]["n_layers"], np.stack([s["vl"] for s in systems]),
        np.stack([s["vr"] for s in systems]), same_leads=same)
    return sysobj, {"uniform_layers": uniform}


def _run_points(systems: list[dict], etas=None, eta_devs=None) -> tuple[np.ndarray, np.ndarray]:
    """T and status for one point per system (each its own k)."""
    dev = _lib.require_cuda()
    sysobj, _ = stack_systems(systems)
    P = len(systems)
    om = torch.tensor([s["omega"] for s in systems], dtype=torch.float64, device=dev)
    et = torch.tensor(etas if etas is not None else [s["eta"] for s in systems], dtype=torch.float64, device=dev)
    ed = torch.tensor(eta_devs if eta_devs is not None else [s["eta_dev"] for s in systems], dtype=torch.float64,
                      device=dev)
    ki = torch.arange(P, dtype=torch.int32, device=dev)
    r = sysobj.transmission(om, ki, et, ed)
    return r["T"].cpu().numpy(), r["status"].cpu().numpy()


def transmission(omega: float, device, lead_left, lead_right, eta: float = 1e-8, eta_device: float | None = None,
                 kpar=None, device_to_lead_left=None, device_to_lead_right=None, contact_left_indices=None,
                 contact_right_indices=None, surface_gf_method: str = "sancho_rubio",
                 omega_scale: float | None = None) -> float:
    """Coherent phonon transmission T(omega) (negfpy ``core/negf.py:306-357``)."""
    check_method(surface_gf_method)
    s = point_system(omega, device, lead_left, lead_right, eta, eta_device, kpar, device_to_lead_left,
                     device_to_lead_right, contact_left_indices, contact_right_indices, omega_scale)
    t, st = _run_points([s])
    raise_for_status(int(st[0]))
    return float(t[0])


def _systems_over_k(omega, device, lead_left, lead_right, kpoints, eta, eta_device, device_to_lead_left,
                    device_to_lead_right, contact_left_indices, contact_right_indices, omega_scale):
    return [point_system(omega, device, lead_left, lead_right, eta, eta_device, k, device_to_lead_left,
                         device_to_lead_right, contact_left_indices, contact_right_indices, omega_scale)
            for k in kpoints]


class _KBatch:
    """All k points of one per-omega call, stacked on the GPU once.

    The blocks of every k come from the GPU builder when the system is a
    material or interface-contact set-up of one parameter set
    (``spectrum._material_fast_path``); otherwise from the per-k host
    builders.  The first k always goes through ``point_system``, which
    validates the call and fixes negfpy's omega-scale and device-eta rules
    (``core/negf.py:163-190``).  ``run`` solves any subset of the k points at
    one ladder eta against the same stack.
    """

    def __init__(self, omega, device, lead_left, lead_right, kpoints, eta_device, device_to_lead_left,
                 device_to_lead_right, contact_left_indices, contact_right_indices, omega_scale):
        from .spectrum import _material_fast_path

        self.K = len(kpoints)
        fast = _material_fast_path(device, lead_left, lead_right, device_to_lead_left, device_to_lead_right,
                                   contact_left_indices, contact_right_indices, omega_scale)
        ks = list(kpoints) if fast is None else list(kpoints[:1])
        systems = _prepare_ladder_systems(omega, device, lead_left, lead_right, ks, eta_device,
                                          device_to_lead_left, device_to_lead_right, contact_left_indices,
                                          contact_right_indices, omega_scale)
        if fast is None:
            self.sys, _ = stack_systems(systems)
        else:
            from .kspace import interface_system, stacked_system

            build = interface_system if fast[0] == "interface" else stacked_system
            self.sys = build(fast[1], fast[2], [() if k is None else k for k in kpoints])
        s0 = systems[0]
        self.omega, self.scale, self.eta_dev_for = s0["omega"], s0["scale"], s0["_eta_dev_for"]

    def run(self, eta: float, idx: list) -> tuple[np.ndarray, np.ndarray]:
        """T and status of the k points ``idx`` at lead eta ``eta`` (before the
        omega scale).  A negative device eta is negfpy's ValueError, i.e. an
        "exception" rejection (status -1, T NaN)."""
        ed = self.eta_dev_for(eta)
        if ed < 0.0:
            return np.full(len(idx), np.nan), np.full(len(idx), -1, dtype=np.int32)
        dev = _lib.require_cuda()
        P = len(idx)
        om = torch.full((P,), float(self.omega), dtype=torch.float64, device=dev)
        et = torch.full((P,), float(eta) / self.scale, dtype=torch.float64, device=dev)
        edt = torch.full((P,), float(ed), dtype=torch.float64, device=dev)
        ki = torch.tensor(list(idx), dtype=torch.int32, device=dev)
        r = self.sys.transmission(om, ki, et, edt)
        return r["T"].cpu().numpy(), r["status"].cpu().numpy()


def transmission_kavg(omega: float, device, lead_left, lead_right, kpoints: list, eta: float = 1e-8,
                      eta_device: float | None = None, device_to_lead_left=None, device_to_lead_right=None,
                      contact_left_indices=None, contact_right_indices=None, surface_gf_method: str = "sancho_rubio",
                      omega_scale: float | None = None) -> float:
    """k-averaged transmission (negfpy ``core/negf.py:360-397``): all k in one batch."""
    if len(kpoints) == 0:
        raise ValueError("kpoints must contain at least one k-point.")
    check_method(surface_gf_method)
    if float(eta if eta_device is None else eta_device) < 0.0:
        raise ValueError("eta_device must be non-negative.")
    kb = _KBatch(omega, device, lead_left, lead_right, kpoints, eta_device, device_to_lead_left,
                 device_to_lead_right, contact_left_indices, contact_right_indices, omega_scale)
    t, st = kb.run(float(eta), list(range(kb.K)))
    for s in st:
        raise_for_status(int(s))
    return float(np.mean(t))


def _check_adaptive_args(kpoints, eta_values, min_success_fraction, nonnegative_tolerance, max_channel_factor):
    """Argument checks shared by the adaptive wrappers (negfpy ``negf.py:423-433``)."""
    if len(kpoints) == 0:
        raise ValueError("kpoints must contain at least one k-point.")
    if len(eta_values) == 0:
        raise ValueError("eta_values must contain at least one eta value.")
    if not (0.0 <= min_success_fraction <= 1.0):
        raise ValueError("min_success_fraction must be in [0, 1].")
    if nonnegative_tolerance < 0.0:
        raise ValueError("nonnegative_tolerance must be non-negative.")
    if max_channel_factor is not None and max_channel_factor <= 0.0:
        raise ValueError("max_channel_factor must be positive when provided.")


def _classify(t, st, max_allowed, nonneg_tol):
    """Reason a point is rejected (None if accepted), in negfpy's order of checks."""
    if st != _lib.OK:
        return "exception"
    if not np.isfinite(t):
        return "non_finite"
    if t < -float(nonneg_tol):
        return "negative"
    if max_allowed is not None and t > max_allowed:
        return "over_channel_limit"
    return None


def _prepare_ladder_systems(omega, device, lead_left, lead_right, kpoints, eta_device, device_to_lead_left,
                            device_to_lead_right, contact_left_indices, contact_right_indices, omega_scale):
    systems = _systems_over_k(omega, device, lead_left, lead_right, kpoints, 1.0, eta_device, device_to_lead_left,
                              device_to_lead_right, contact_left_indices, contact_right_indices, omega_scale)
    scale = 1.0 if omega_scale is None else float(omega_scale)
    for s in systems:
        s["scale"] = scale
        if eta_device is None:
            s["_eta_dev_for"] = (lambda sc: (lambda e: e / sc))(scale)
        else:
            fixed = float(eta_device) / scale
            s["_eta_dev_for"] = (lambda v: (lambda e: v))(fixed)
    return systems


def transmission_kavg_adaptive(omega: float, device, lead_left, lead_right, kpoints: list,
                               eta_values: tuple = (1e-8, 1e-7, 1e-6, 1e-5), eta_device: float | None = None,
                               min_success_fraction: float = 0.0, device_to_lead_left=None,
                               device_to_lead_right=None, contact_left_indices=None, contact_right_indices=None,
                               surface_gf_method: str = "sancho_rubio", omega_scale: float | None = None,
                               nonnegative_tolerance: float = 0.0, max_channel_factor: float | None = None,
                               collect_rejected: bool = False) -> tuple[float, dict]:
    """Per-k eta ladder (negfpy ``core/negf.py:400-543``), one batch per ladder rung.

    Points that fail at one eta are re-launched together at the next one;
    results, statistics and the rejected list are those of negfpy's per-k
    loop (the rejected list is returned in the same k-major order).
    """
    _check_adaptive_args(kpoints, eta_values, min_success_fraction, nonnegative_tolerance, max_channel_factor)
    check_method(surface_gf_method)
    kb = _KBatch(omega, device, lead_left, lead_right, kpoints, eta_device, device_to_lead_left,
                 device_to_lead_right, contact_left_indices, contact_right_indices, omega_scale)
    K = len(kpoints)
    # one call shares the lead order over its k points (stack_systems checks it)
    max_allowed = [None if max_channel_factor is None else float(max_channel_factor) * float(kb.sys.nl)] * K
    accepted: dict[int, tuple[float, float]] = {}
    attempts: list[tuple[int, int, dict]] = []
    pending = list(range(K))
    for ei, eta in enumerate(eta_values):
        if not pending:
            break
        t, st = kb.run(float(eta), pending)
        nxt = []
        for j, ki in enumerate(pending):
            reason = _classify(t[j], st[j], max_allowed[ki], nonnegative_tolerance)
            if reason is None:
                accepted[ki] = (float(max(t[j], 0.0)), float(eta))
            else:
                kp = kpoints[ki]
                attempts.append((ki, ei, {"omega": float(omega),
                                          "kpar": tuple(float(x) for x in kp) if kp is not None else (),
                                          "eta": float(eta), "t": None if reason == "exception" else float(t[j]),
                                          "reason": reason}))
                nxt.append(ki)
        pending = nxt
    vals = [accepted[i][0] for i in range(K) if i in accepted]
    used = [accepted[i][1] for i in range(K) if i in accepted]
    n_success = len(vals)
    success_fraction = float(n_success / K)
    if n_success == 0:
        raise RuntimeError("No k-point converged for adaptive k-averaged transmission.")
    if success_fraction < min_success_fraction:
        raise RuntimeError(
            "Adaptive k-averaged transmission failed success-fraction threshold "
            f"(got {success_fraction:.3f}, required >= {min_success_fraction:.3f}).")
    info = {
        "n_total": int(K),
        "n_success": int(n_success),
        "n_failed": int(K - n_success),
        "success_fraction": success_fraction,
        "eta_histogram": {float(e): int(sum(1 for u in used if u == float(e))) for e in eta_values},
    }
    if collect_rejected:
        rej = [a[2] for a in sorted(attempts, key=lambda a: (a[0], a[1]))]
        info["n_rejected"] = len(rej)
        info["rejected"] = rej
    return float(np.mean(vals)), info


def transmission_kavg_adaptive_global_eta(omega: float, device, lead_left, lead_right, kpoints: list,
                                          eta_values: tuple = (1e-8, 1e-7, 1e-6, 1e-5),
                                          eta_device: float | None = None, min_success_fraction: float = 0.0,
                                          device_to_lead_left=None, device_to_lead_right=None,
                                          contact_left_indices=None, contact_right_indices=None,
                                          surface_gf_method: str = "sancho_rubio",
                                          omega_scale: float | None = None, nonnegative_tolerance: float = 0.0,
                                          max_channel_factor: float | None = None,
                                          collect_rejected: bool = False) -> tuple[float, dict]:
    """One eta per omega (negfpy ``core/negf.py:546-688``): all k per rung in one batch."""
    _check_adaptive_args(kpoints, eta_values, min_success_fraction, nonnegative_tolerance, max_channel_factor)
    check_method(surface_gf_method)
    kb = _KBatch(omega, device, lead_left, lead_right, kpoints, eta_device, device_to_lead_left,
                 device_to_lead_right, contact_left_indices, contact_right_indices, omega_scale)
    K = len(kpoints)
    # one call shares the lead order over its k points (stack_systems checks it)
    max_allowed = [None if max_channel_factor is None else float(max_channel_factor) * float(kb.sys.nl)] * K
    rejected_all: list = []
    for eta in eta_values:
        t, st = kb.run(float(eta), list(range(K)))
        vals = []
        for ki in range(K):
            reason = _classify(t[ki], st[ki], max_allowed[ki], nonnegative_tolerance)
            if reason is None:
                vals.append(float(max(t[ki], 0.0)))
            elif collect_rejected:
                kp = kpoints[ki]
                rejected_all.append({"omega": float(omega),
                                     "kpar": tuple(float(x) for x in kp) if kp is not None else (),
                                     "eta": float(eta), "t": None if reason == "exception" else float(t[ki]),
                                     "reason": reason})
        n_success = len(vals)
        success_fraction = float(n_success / K)
        if n_success > 0 and success_fraction >= min_success_fraction:
            info = {
                "n_total": int(K),
                "n_success": int(n_success),
                "n_failed": int(K - n_success),
                "success_fraction": success_fraction,
                "eta_selected": float(eta),
                "eta_histogram": {float(e): (int(n_success) if float(e) == float(eta) else 0) for e in eta_values},
            }
            if collect_rejected:
                info["n_rejected"] = int(len(rejected_all))
                info["rejected"] = rejected_all
            return float(np.mean(vals)), info
    raise RuntimeError(
        "No eta value satisfied global adaptive k-averaging quality threshold "
        f"(required success_fraction >= {min_success_fraction:.3f}).")


def device_green_function(omega: float, device, lead_left, lead_right, eta: float = 1e-8,
                          eta_device: float | None = None, kpar=None, device_to_lead_left=None,
                          device_to_lead_right=None, contact_left_indices=None, contact_right_indices=None,
                          surface_gf_method: str = "sancho_rubio", omega_scale: float | None = None):
    """(G, Sigma_L, Sigma_R) of the finite device (negfpy ``core/negf.py:253-303``).

    G is the dense (L n) x (L n) inverse of A = (omega + i eta_d)^2 - D - Sigma,
    every block computed on the GPU by a left-connected sweep and backward
    recursions (``negf_device_green_f64``); Sigma_L and Sigma_R are embedded in
    (L n) x (L n) matrices at the contact indices, as negfpy returns them.  The
    contacts must lie in the first / last principal layer (``ValueError``
    otherwise, as for ``transmission``)."""
    check_method(surface_gf_method)
    dev = _lib.require_cuda()
    s = point_system(omega, device, lead_left, lead_right, eta, eta_device, kpar, device_to_lead_left,
                     device_to_lead_right, contact_left_indices, contact_right_indices, omega_scale)
    sysobj, _ = stack_systems([s])
    om = torch.tensor([s["omega"]], dtype=torch.float64, device=dev)
    et = torch.tensor([s["eta"]], dtype=torch.float64, device=dev)
    ed = torch.tensor([s["eta_dev"]], dtype=torch.float64, device=dev)
    ki = torch.zeros(1, dtype=torch.int32, device=dev)
    rl = engine.sgf_sr(*sysobj.lead_l, om, et, ki)
    rr = rl if sysobj.same_leads else engine.sgf_sr(*sysobj.lead_r, om, et, ki)
    lst = torch.where(rl["status"] != 0, rl["status"], rr["status"])
    G, sl, sr, st = engine.device_green(sysobj.onsite, sysobj.coupling, sysobj.n_layers, sysobj.vl, sysobj.vr,
                                        rl["g"], rr["g"], om, ed, ki, lst)
    raise_for_status(int(st[0]))
    n = sysobj.n
    dim = sysobj.n_layers * n
    sigma_l = np.zeros((dim, dim), dtype=np.complex128)
    sigma_r = np.zeros((dim, dim), dtype=np.complex128)
    sigma_l[:n, :n] = sl[0].cpu().numpy()
    sigma_r[dim - n:, dim - n:] = sr[0].cpu().numpy()
    return G[0].cpu().numpy(), sigma_l, sigma_r
