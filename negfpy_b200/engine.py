"""Batched device-side engine: stacked blocks on the GPU, one launch per stage.

A *point* is one (omega, k) pair.  Blocks are stacked per k once
(``[K, n, n]`` for lead blocks, ``[K, L or 1, n, n]`` for the device) and
every point carries its k index, so a frequency sweep never rebuilds or
re-uploads blocks.  Stages per chunk of points:

1. ``negf_sgf_sr_f64`` for the left lead (and the right lead unless both
   leads are the same object, in which case its result is reused),
2. ``negf_rgf_transmission_f64`` for Sigma, the RGF sweep and the trace.

All tensors are complex128/float64 on the current CUDA device.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _lib

CDT = torch.complex128
RDT = torch.float64


def _dev() -> torch.device:
    return _lib.require_cuda()


def _c(t, device=None) -> torch.Tensor:
    t = torch.as_tensor(np.asarray(t) if not isinstance(t, torch.Tensor) else t)
    return t.to(device=device or _dev(), dtype=CDT).contiguous()


def _r(t, device=None) -> torch.Tensor:
    t = torch.as_tensor(t) if not isinstance(t, torch.Tensor) else t
    return t.to(device=device or _dev(), dtype=RDT).contiguous()


def sgf_sr(d00: torch.Tensor, d01: torch.Tensor, d10: torch.Tensor | None, omega: torch.Tensor, eta: torch.Tensor,
           k_index: torch.Tensor | None = None, tol: float = 1e-12, maxiter: int = 200, want_g: bool = True,
           want_dos: bool = False, stream=None) -> dict:
    """Sancho-Rubio surface GF for P points over K stacked lead sets ``[K, n, n]``."""
    lib = _lib.load()
    dev = _dev()
    if d00.dim() == 2:
        d00, d01 = d00[None], d01[None]
        d10 = None if d10 is None else d10[None]
    K, n, _ = d00.shape
    P = int(omega.shape[0])
    g = torch.empty((P, n, n), dtype=CDT, device=dev) if want_g else None
    dos = torch.empty(P, dtype=RDT, device=dev) if want_dos else None
    iters = torch.empty(P, dtype=torch.int32, device=dev)
    status = torch.empty(P, dtype=torch.int32, device=dev)
    if P == 0:
        return {"g": g, "dos": dos, "iters": iters, "status": status}
    if k_index is not None:
        k_index = k_index.to(device=dev, dtype=torch.int32).contiguous()
    need = int(lib.negf_sgf_workspace_bytes(n))
    if need == 0:
        raise RuntimeError(f"block order {n} is not supported by the FP64 kernels")
    ws = _workspace(need, dev, "sgf")
    rc = lib.negf_sgf_sr_f64(n, P, _lib.ptr(d00), _lib.ptr(d01), _lib.ptr(d10), n * n if K > 1 else 0,
                             _lib.ptr(k_index), _lib.ptr(omega), _lib.ptr(eta), float(tol), int(maxiter),
                             _lib.ptr(g), _lib.ptr(dos), _lib.ptr(iters), _lib.ptr(status), _lib.ptr(ws),
                             ws.numel(), _lib.stream_handle(stream))
    _lib.check(rc, "negf_sgf_sr_f64")
    return {"g": g, "dos": dos, "iters": iters, "status": status}


_ws_cache: dict = {}


def _workspace(nbytes: int, dev: torch.device, role: str = "rgf") -> torch.Tensor:
    """Cached device workspace per (device, role); grown on demand.  Calls on
    one stream reuse it safely (each launch resets its own work counter)."""
    key = (dev.index, role)
    t = _ws_cache.get(key)
    if t is None or t.numel() < nbytes:
        t = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=dev)
        _ws_cache[key] = t
    return t


def rgf_transmission(onsite: torch.Tensor, coupling: torch.Tensor | None, n_layers: int, vl: torch.Tensor,
                     vr: torch.Tensor, gl: torch.Tensor, gr: torch.Tensor, omega: torch.Tensor,
                     eta_dev: torch.Tensor, k_index: torch.Tensor | None, lead_status: torch.Tensor | None,
                     stream=None, precision: str = "f64") -> tuple[torch.Tensor, torch.Tensor]:
    """T for P points.  ``onsite`` ``[K, L|1, n, n]``, ``coupling`` ``[K, L-1|1, n, n]``,
    ``vl`` ``[K|1, n, nl]``, ``vr`` ``[K|1, n, nr]``, ``gl`` ``[P, nl, nl]``, ``gr`` ``[P, nr, nr]``.

    ``precision``: "f64" (``negf_rgf_transmission_f64``) or "mixed"
    (``negf_rgf_transmission_mixed``: FP32 sweep, FP64 self-energies and trace;
    no fallback here, failed points keep their status)."""
    if precision not in ("f64", "mixed"):
        raise ValueError(f"unknown precision {precision!r}; expected 'f64' or 'mixed'")
    lib = _lib.load()
    dev = _dev()
    K, Lo, n, _ = onsite.shape
    nl, nr = int(vl.shape[-1]), int(vr.shape[-1])
    P = int(omega.shape[0])
    T = torch.empty(P, dtype=RDT, device=dev)
    st = torch.empty(P, dtype=torch.int32, device=dev)
    if P == 0:
        return T, st
    on_ks = Lo * n * n if K > 1 else 0
    on_ls = 0 if Lo == 1 else n * n
    if coupling is None or n_layers == 1:
        cp, cp_ks, cp_ls = None, 0, 0
    else:
        Kc, Lc = coupling.shape[0], coupling.shape[1]
        cp, cp_ks, cp_ls = coupling, (Lc * n * n if Kc > 1 else 0), (0 if Lc == 1 else n * n)
    vl_ks = n * nl if vl.shape[0] > 1 else 0
    vr_ks = n * nr if vr.shape[0] > 1 else 0
    mixed = precision == "mixed"
    need = int(lib.negf_rgf_mixed_workspace_bytes(n, nl, nr) if mixed else lib.negf_rgf_workspace_bytes(n, nl, nr))
    if need == 0:
        raise RuntimeError(f"block order {max(n, nl, nr)} is not supported by the {precision} kernels")
    ws = _workspace(need, dev, "rgf_mixed" if mixed else "rgf")
    if k_index is not None:
        k_index = k_index.to(device=dev, dtype=torch.int32).contiguous()
    fn = lib.negf_rgf_transmission_mixed if mixed else lib.negf_rgf_transmission_f64
    rc = fn(
        n, nl, nr, int(n_layers), P, _lib.ptr(onsite), on_ks, on_ls, _lib.ptr(cp), cp_ks, cp_ls, _lib.ptr(vl), vl_ks,
        _lib.ptr(vr), vr_ks, _lib.ptr(gl), nl * nl, _lib.ptr(gr), nr * nr, _lib.ptr(k_index), _lib.ptr(omega),
        _lib.ptr(eta_dev), _lib.ptr(lead_status), _lib.ptr(T), _lib.ptr(st), _lib.ptr(ws), ws.numel(),
        _lib.stream_handle(stream))
    _lib.check(rc, "negf_rgf_transmission_mixed" if mixed else "negf_rgf_transmission_f64")
    return T, st


REFINE_TOL = 1e-12
REFINE_MAX_STEPS = 5


def rgf_transmission_refine64(onsite, coupling, n_layers, vl, vr, gl, gr, omega, eta_dev, k_index, lead_status,
                              stream=None, tol: float = REFINE_TOL, max_steps: int = REFINE_MAX_STEPS):
    """T, status and refinement steps for P points from FP32 factors refined
    to FP64 accuracy (``negf_rgf_transmission_refined``); blocks as in
    ``rgf_transmission``.  Points that do not converge report
    ``_lib.REFINE_FAIL`` (no fallback here)."""
    lib = _lib.load()
    dev = _dev()
    K, Lo, n, _ = onsite.shape
    nl, nr = int(vl.shape[-1]), int(vr.shape[-1])
    P = int(omega.shape[0])
    T = torch.empty(P, dtype=RDT, device=dev)
    st = torch.empty(P, dtype=torch.int32, device=dev)
    steps = torch.zeros(P, dtype=torch.int32, device=dev)
    if P == 0:
        return T, st, steps
    on_ks = Lo * n * n if K > 1 else 0
    on_ls = 0 if Lo == 1 else n * n
    if coupling is None or n_layers == 1:
        cp, cp_ks, cp_ls = None, 0, 0
    else:
        Kc, Lc = coupling.shape[0], coupling.shape[1]
        cp, cp_ks, cp_ls = coupling, (Lc * n * n if Kc > 1 else 0), (0 if Lc == 1 else n * n)
    need = int(lib.negf_rgf_refined_workspace_bytes(n, nl, nr, int(n_layers)))
    if need == 0:
        raise RuntimeError(f"block order {max(n, nl, nr)} is not supported by the refined kernel")
    ws = _workspace(need, dev, "rgf_refined")
    if k_index is not None:
        k_index = k_index.to(device=dev, dtype=torch.int32).contiguous()
    rc = lib.negf_rgf_transmission_refined(
        n, nl, nr, int(n_layers), P, _lib.ptr(onsite), on_ks, on_ls, _lib.ptr(cp), cp_ks, cp_ls, _lib.ptr(vl),
        n * nl if vl.shape[0] > 1 else 0, _lib.ptr(vr), n * nr if vr.shape[0] > 1 else 0, _lib.ptr(gl), nl * nl,
        _lib.ptr(gr), nr * nr, _lib.ptr(k_index), _lib.ptr(omega), _lib.ptr(eta_dev), _lib.ptr(lead_status),
        float(tol), int(max_steps), _lib.ptr(T), _lib.ptr(st), _lib.ptr(steps), _lib.ptr(ws), ws.numel(),
        _lib.stream_handle(stream))
    _lib.check(rc, "negf_rgf_transmission_refined")
    return T, st, steps


def _fallback_f64(T, st, onsite, coupling, n_layers, vl, vr, gl, gr, omega, eta_dev, k_index, lead_status, stream):
    """Re-solve in FP64 the points whose reduced-precision solve failed while
    their leads succeeded; returns the number re-solved."""
    bad = st != 0
    if lead_status is not None:
        bad &= lead_status == 0
    idx = torch.nonzero(bad).flatten()
    nbad = int(idx.numel())
    if nbad:
        ki = None if k_index is None else k_index[idx]
        t2, s2 = rgf_transmission(onsite, coupling, n_layers, vl, vr, gl[idx].contiguous(), gr[idx].contiguous(),
                                  omega[idx].contiguous(), eta_dev[idx].contiguous(), ki, None, stream)
        T[idx] = t2
        st[idx] = s2
    return nbad


def rgf_transmission_refined(onsite, coupling, n_layers, vl, vr, gl, gr, omega, eta_dev, k_index, lead_status,
                             stream=None, tol: float = REFINE_TOL, max_steps: int = REFINE_MAX_STEPS):
    """Refined device solve with an FP64 fallback: FP32 factors and FP64
    iterative refinement (``rgf_transmission_refine64``); the points that
    report NEGF_REFINE_FAIL, or a singular / non-finite FP32 pivot, while
    their leads succeeded are solved again by the FP64 kernel.  Returns
    (T, status, number re-solved, refinement steps per point)."""
    T, st, steps = rgf_transmission_refine64(onsite, coupling, n_layers, vl, vr, gl, gr, omega, eta_dev, k_index,
                                             lead_status, stream, tol, max_steps)
    nbad = _fallback_f64(T, st, onsite, coupling, n_layers, vl, vr, gl, gr, omega, eta_dev, k_index, lead_status,
                         stream)
    return T, st, nbad, steps


def rgf_transmission_mixed(onsite, coupling, n_layers, vl, vr, gl, gr, omega, eta_dev, k_index, lead_status,
                           stream=None) -> tuple[torch.Tensor, torch.Tensor, int]:
    """Mixed-precision device solve (FP32 sweep, no refinement) with an FP64
    fallback: points whose FP32 sweep failed (singular or non-finite pivot)
    while their leads succeeded are solved again by the FP64 kernel.  Returns
    (T, status, number re-solved)."""
    T, st = rgf_transmission(onsite, coupling, n_layers, vl, vr, gl, gr, omega, eta_dev, k_index, lead_status,
                             stream, precision="mixed")
    bad = st != 0
    if lead_status is not None:
        bad &= lead_status == 0
    idx = torch.nonzero(bad).flatten()
    nbad = int(idx.numel())
    if nbad:
        ki = None if k_index is None else k_index[idx]
        t2, s2 = rgf_transmission(onsite, coupling, n_layers, vl, vr, gl[idx].contiguous(), gr[idx].contiguous(),
                                  omega[idx].contiguous(), eta_dev[idx].contiguous(), ki, None, stream)
        T[idx] = t2
        st[idx] = s2
    return T, st, nbad


def device_green(onsite: torch.Tensor, coupling: torch.Tensor | None, n_layers: int, vl: torch.Tensor,
                 vr: torch.Tensor, gl: torch.Tensor, gr: torch.Tensor, omega: torch.Tensor, eta_dev: torch.Tensor,
                 k_index: torch.Tensor | None, lead_status: torch.Tensor | None, stream=None):
    """Full device G ``[P, L n, L n]`` and Sigma_L, Sigma_R ``[P, n, n]`` with status
    (``negf_device_green_f64``); blocks as in ``rgf_transmission``."""
    lib = _lib.load()
    dev = _dev()
    K, Lo, n, _ = onsite.shape
    nl, nr = int(vl.shape[-1]), int(vr.shape[-1])
    P = int(omega.shape[0])
    dim = int(n_layers) * n
    G = torch.empty((P, dim, dim), dtype=CDT, device=dev)
    sl = torch.empty((P, n, n), dtype=CDT, device=dev)
    sr = torch.empty((P, n, n), dtype=CDT, device=dev)
    st = torch.empty(P, dtype=torch.int32, device=dev)
    if P == 0:
        return G, sl, sr, st
    on_ks = Lo * n * n if K > 1 else 0
    on_ls = 0 if Lo == 1 else n * n
    if coupling is None or n_layers == 1:
        cp, cp_ks, cp_ls = None, 0, 0
    else:
        Kc, Lc = coupling.shape[0], coupling.shape[1]
        cp, cp_ks, cp_ls = coupling, (Lc * n * n if Kc > 1 else 0), (0 if Lc == 1 else n * n)
    need = int(lib.negf_device_green_workspace_bytes(n, nl, nr, int(n_layers)))
    if need == 0:
        raise RuntimeError(f"block order {max(n, nl, nr)} is not supported by the device Green's function kernel")
    ws = _workspace(need, dev, "device_green")
    if k_index is not None:
        k_index = k_index.to(device=dev, dtype=torch.int32).contiguous()
    rc = lib.negf_device_green_f64(
        n, nl, nr, int(n_layers), P, _lib.ptr(onsite), on_ks, on_ls, _lib.ptr(cp), cp_ks, cp_ls, _lib.ptr(vl),
        n * nl if vl.shape[0] > 1 else 0, _lib.ptr(vr), n * nr if vr.shape[0] > 1 else 0, _lib.ptr(gl), nl * nl,
        _lib.ptr(gr), nr * nr, _lib.ptr(k_index), _lib.ptr(omega), _lib.ptr(eta_dev), _lib.ptr(lead_status),
        _lib.ptr(G), _lib.ptr(sl), _lib.ptr(sr), _lib.ptr(st), _lib.ptr(ws), ws.numel(), _lib.stream_handle(stream))
    _lib.check(rc, "negf_device_green_f64")
    return G, sl, sr, st


# Per-point gradient blocks are produced in chunks of at most this many bytes
# (large chunks keep the persistent adjoint launches full).
_POINTS_CHUNK_BYTES = 8 << 30


def _sum_by_k(dst: torch.Tensor, src: torch.Tensor, kidx: torch.Tensor | None) -> None:
    """dst[k] += the sum of src[p] over the points p with kidx[p] == k, each
    k's points summed by one reduction in point order (no atomics), so the
    result is the same bit for bit from run to run.  kidx None: all into
    dst[0]."""
    if src.shape[0] == 0:
        return
    if kidx is None or dst.shape[0] == 1:
        dst[0] += src.sum(0)
        return
    kk = kidx.to(torch.int64)
    order = torch.argsort(kk, stable=True)
    uniq, counts = torch.unique_consecutive(kk[order], return_counts=True)
    start = 0
    for k, c in zip(uniq.tolist(), counts.tolist()):
        dst[k] += src[order[start:start + c]].sum(0)
        start += c


def rgf_adjoint(onsite: torch.Tensor, coupling: torch.Tensor, n_layers: int, vl: torch.Tensor, vr: torch.Tensor,
                gl: torch.Tensor, gr: torch.Tensor, omega: torch.Tensor, eta_dev: torch.Tensor,
                k_index: torch.Tensor, lead_status: torch.Tensor | None, weight: torch.Tensor,
                stream=None, want_sigma: bool = False, deterministic: bool = False):
    """Vector-Jacobian product of T with respect to the device blocks.

    Layer-resolved blocks ``onsite`` ``[K, L, n, n]`` and ``coupling`` ``[K, L-1, n, n]``
    (no stride-0 sharing: every block is a variable).  Returns (T, status,
    grad_onsite, grad_coupling) with sum_p weight[p] dT_p = 2 Re sum Tr[dD X]
    over the returned adjoint blocks (``negf_rgf_adjoint_f64``).  With
    ``want_sigma`` it also returns the per-point weighted adjoints of the two
    contact self-energies ``[P, n, n]`` (``negf_rgf_adjoint_sigma_f64``), the
    input of ``sgf_adjoint``.

    ``deterministic``: the points store their blocks separately
    (``negf_rgf_adjoint_points_f64``, in chunks of at most 8 GiB) and the
    blocks are summed per k in a fixed order, so the gradient is the same
    bit for bit from run to run (the default adds them with FP64 atomics)."""
    lib = _lib.load()
    dev = _dev()
    K, L, n, _ = onsite.shape
    if L != n_layers:
        raise ValueError("rgf_adjoint needs one onsite block per layer")
    nl, nr = int(vl.shape[-1]), int(vr.shape[-1])
    P = int(omega.shape[0])
    T = torch.empty(P, dtype=RDT, device=dev)
    st = torch.empty(P, dtype=torch.int32, device=dev)
    g_on = torch.zeros((K, L, n, n), dtype=CDT, device=dev)
    g_cp = torch.zeros((K, max(L - 1, 1), n, n), dtype=CDT, device=dev)
    xs_l = torch.zeros((P, n, n), dtype=CDT, device=dev) if want_sigma else None
    xs_r = torch.zeros((P, n, n), dtype=CDT, device=dev) if want_sigma else None
    if P == 0:
        return (T, st, g_on, g_cp, xs_l, xs_r) if want_sigma else (T, st, g_on, g_cp)
    if L > 1 and (coupling is None or tuple(coupling.shape) != (K, L - 1, n, n)):
        raise ValueError("rgf_adjoint needs coupling blocks [K, L-1, n, n]")
    need = int(lib.negf_adjoint_workspace_bytes(n, nl, nr, L))
    if need == 0:
        raise RuntimeError(f"block order {max(n, nl, nr)} is not supported by the adjoint kernel")
    ws = _workspace(need, dev, "adjoint")
    k_index = k_index.to(device=dev, dtype=torch.int32).contiguous()
    vl_ks = n * nl if vl.shape[0] > 1 else 0
    vr_ks = n * nr if vr.shape[0] > 1 else 0
    cp = coupling if L > 1 else None
    common = (n, nl, nr, L, P, _lib.ptr(onsite), L * n * n, n * n, _lib.ptr(cp), (L - 1) * n * n, n * n,
              _lib.ptr(vl), vl_ks, _lib.ptr(vr), vr_ks, _lib.ptr(gl), nl * nl, _lib.ptr(gr), nr * nr,
              _lib.ptr(k_index), _lib.ptr(omega), _lib.ptr(eta_dev), _lib.ptr(lead_status), _lib.ptr(weight),
              _lib.ptr(g_on), _lib.ptr(g_cp if L > 1 else None))
    tail = (_lib.ptr(T), _lib.ptr(st), _lib.ptr(ws), ws.numel(), _lib.stream_handle(stream))
    if deterministic:
        weight = weight.to(device=dev, dtype=RDT).contiguous()
        lst = None if lead_status is None else lead_status.to(device=dev, dtype=torch.int32).contiguous()
        chunk = max(1, min(P, _POINTS_CHUNK_BYTES // ((2 * L - 1) * n * n * 16)))
        pp_on = torch.empty((chunk, L, n, n), dtype=CDT, device=dev)
        pp_cp = torch.empty((chunk, max(L - 1, 1), n, n), dtype=CDT, device=dev)
        for a in range(0, P, chunk):
            b = min(P, a + chunk)
            c = b - a
            pp_on[:c].zero_()
            pp_cp[:c].zero_()
            sl = slice(a, b)
            rc = lib.negf_rgf_adjoint_points_f64(
                n, nl, nr, L, c, _lib.ptr(onsite), L * n * n, n * n, _lib.ptr(cp), (L - 1) * n * n, n * n,
                _lib.ptr(vl), vl_ks, _lib.ptr(vr), vr_ks, _lib.ptr(gl[sl]), nl * nl, _lib.ptr(gr[sl]), nr * nr,
                _lib.ptr(k_index[sl]), _lib.ptr(omega[sl]), _lib.ptr(eta_dev[sl]),
                _lib.ptr(None if lst is None else lst[sl]), _lib.ptr(weight[sl]), _lib.ptr(pp_on),
                _lib.ptr(pp_cp if L > 1 else None), _lib.ptr(None if xs_l is None else xs_l[sl]),
                _lib.ptr(None if xs_r is None else xs_r[sl]), _lib.ptr(T[sl]), _lib.ptr(st[sl]), _lib.ptr(ws),
                ws.numel(), _lib.stream_handle(stream))
            _lib.check(rc, "negf_rgf_adjoint_points_f64")
            _sum_by_k(g_on, pp_on[:c], k_index[sl])
            if L > 1:
                _sum_by_k(g_cp, pp_cp[:c], k_index[sl])
        return (T, st, g_on, g_cp, xs_l, xs_r) if want_sigma else (T, st, g_on, g_cp)
    if want_sigma:
        rc = lib.negf_rgf_adjoint_sigma_f64(*common, _lib.ptr(xs_l), _lib.ptr(xs_r), *tail)
        _lib.check(rc, "negf_rgf_adjoint_sigma_f64")
        return T, st, g_on, g_cp, xs_l, xs_r
    rc = lib.negf_rgf_adjoint_f64(*common, *tail)
    _lib.check(rc, "negf_rgf_adjoint_f64")
    return T, st, g_on, g_cp


def sgf_adjoint(d01: torch.Tensor, d10: torch.Tensor | None, v: torch.Tensor, g: torch.Tensor,
                sigma_adj: torch.Tensor, k_index: torch.Tensor | None, lead_status: torch.Tensor | None = None,
                tol: float = 1e-12, maxiter: int = 200, stream=None, deterministic: bool = False) -> dict:
    """Adjoint of the lead surface GF and of Sigma = V g V^H (``negf_sgf_adjoint_f64``).

    ``d01``/``d10`` ``[K, nl, nl]`` (d10 None: d01^H), ``v`` ``[K|1, n, nl]``,
    ``g`` ``[P, nl, nl]`` the surface GFs, ``sigma_adj`` ``[P, n, n]`` the
    weighted self-energy adjoints of ``rgf_adjoint(want_sigma=True)``.
    Returns the per-k adjoint blocks (dT = 2 Re Tr[dH X]) ``h00``, ``h01``,
    ``h10`` (None when d10 is None: its part is folded into ``h01``) of shape
    ``[K, nl, nl]``, ``v`` of shape ``[K|1, nl, n]``, and per-point
    ``iters``/``status``.  ``deterministic``: per-point terms
    (``negf_sgf_adjoint_points_f64``) summed per k in a fixed order, the same
    bit for bit from run to run (the default adds them with FP64 atomics)."""
    lib = _lib.load()
    dev = _dev()
    if d01.dim() == 2:
        d01 = d01[None]
        d10 = None if d10 is None else d10[None]
    K, nl, _ = d01.shape
    n = int(v.shape[-2])
    P = int(g.shape[0])
    gh00 = torch.zeros((K, nl, nl), dtype=CDT, device=dev)
    gh01 = torch.zeros((K, nl, nl), dtype=CDT, device=dev)
    gh10 = None if d10 is None else torch.zeros((K, nl, nl), dtype=CDT, device=dev)
    gv = torch.zeros((v.shape[0], nl, n), dtype=CDT, device=dev)
    iters = torch.zeros(P, dtype=torch.int32, device=dev)
    status = torch.zeros(P, dtype=torch.int32, device=dev)
    out = {"h00": gh00, "h01": gh01, "h10": gh10, "v": gv, "iters": iters, "status": status}
    if P == 0:
        return out
    need = int(lib.negf_sgf_adjoint_workspace_bytes(nl, n))
    if need == 0:
        raise RuntimeError(f"block order {max(nl, n)} is not supported by the surface-GF adjoint kernel")
    ws = _workspace(need, dev, "sgf_adjoint")
    if k_index is not None:
        k_index = k_index.to(device=dev, dtype=torch.int32).contiguous()
    if deterministic:
        d01c = d01.contiguous()
        d10c = None if d10 is None else d10.contiguous()
        vc, gc, xc = v.contiguous(), g.contiguous(), sigma_adj.contiguous()
        lst = None if lead_status is None else lead_status.to(device=dev, dtype=torch.int32).contiguous()
        per = (3 * nl * nl + nl * n) * 16
        chunk = max(1, min(P, _POINTS_CHUNK_BYTES // per))
        p00 = torch.empty((chunk, nl, nl), dtype=CDT, device=dev)
        p01 = torch.empty((chunk, nl, nl), dtype=CDT, device=dev)
        p10 = None if d10 is None else torch.empty((chunk, nl, nl), dtype=CDT, device=dev)
        pv = torch.empty((chunk, nl, n), dtype=CDT, device=dev)
        for a in range(0, P, chunk):
            b = min(P, a + chunk)
            c = b - a
            sl = slice(a, b)
            for t in (p00, p01, p10, pv):
                if t is not None:
                    t[:c].zero_()
            rc = lib.negf_sgf_adjoint_points_f64(
                nl, n, c, _lib.ptr(d01c), _lib.ptr(d10c), nl * nl if K > 1 else 0, _lib.ptr(vc),
                n * nl if v.shape[0] > 1 else 0, _lib.ptr(gc[sl]), nl * nl, _lib.ptr(xc[sl]),
                _lib.ptr(None if k_index is None else k_index[sl]), _lib.ptr(None if lst is None else lst[sl]),
                float(tol), int(maxiter), _lib.ptr(p00), _lib.ptr(p01), _lib.ptr(p10), _lib.ptr(pv),
                _lib.ptr(iters[sl]), _lib.ptr(status[sl]), _lib.ptr(ws), ws.numel(), _lib.stream_handle(stream))
            _lib.check(rc, "negf_sgf_adjoint_points_f64")
            ks = None if k_index is None else k_index[sl]
            _sum_by_k(gh00, p00[:c], ks)
            _sum_by_k(gh01, p01[:c], ks)
            if gh10 is not None:
                _sum_by_k(gh10, p10[:c], ks)
            _sum_by_k(gv, pv[:c], ks)
        return out
    rc = lib.negf_sgf_adjoint_f64(nl, n, P, _lib.ptr(d01.contiguous()), _lib.ptr(None if d10 is None else
                                                                                d10.contiguous()),
                                  nl * nl if K > 1 else 0, _lib.ptr(v.contiguous()), n * nl if v.shape[0] > 1 else 0,
                                  _lib.ptr(g.contiguous()), nl * nl, _lib.ptr(sigma_adj.contiguous()),
                                  _lib.ptr(k_index), _lib.ptr(lead_status), float(tol), int(maxiter),
                                  _lib.ptr(gh00), _lib.ptr(gh01), _lib.ptr(gh10), _lib.ptr(gv), _lib.ptr(iters),
                                  _lib.ptr(status), _lib.ptr(ws), ws.numel(), _lib.stream_handle(stream))
    _lib.check(rc, "negf_sgf_adjoint_f64")
    return out


def kavg(T_wk: torch.Tensor, stream=None) -> torch.Tensor:
    """Mean over k of an omega-major ``[W, K]`` table."""
    lib = _lib.load()
    W, K = T_wk.shape
    out = torch.empty(W, dtype=RDT, device=T_wk.device)
    _lib.check(lib.negf_kavg_f64(_lib.ptr(T_wk.contiguous()), W, K, _lib.ptr(out), _lib.stream_handle(stream)),
               "negf_kavg_f64")
    return out


def kappa(omega: torch.Tensor, tbar: torch.Tensor, temperatures, omega_unit_rad_s: float, stream=None) -> torch.Tensor:
    lib = _lib.load()
    temps = _r(torch.as_tensor(np.atleast_1d(np.asarray(temperatures, dtype=float))), omega.device)
    out = torch.empty(temps.shape[0], dtype=RDT, device=omega.device)
    _lib.check(lib.negf_kappa_f64(_lib.ptr(omega), _lib.ptr(tbar), int(omega.shape[0]), _lib.ptr(temps),
                                  int(temps.shape[0]), float(omega_unit_rad_s), _lib.ptr(out),
                                  _lib.stream_handle(stream)), "negf_kappa_f64")
    return out


@dataclass
class StackedSystem:
    """Device-resident blocks of one lead/device/lead system over K k-points."""

    lead_l: tuple  # (d00, d01, d10|None) [K, nl, nl]
    lead_r: tuple
    onsite: torch.Tensor  # [K, L|1, n, n]
    coupling: torch.Tensor | None  # [K, L-1|1, n, n]
    n_layers: int
    vl: torch.Tensor  # [K|1, n, nl]
    vr: torch.Tensor  # [K|1, n, nr]
    same_leads: bool

    @property
    def n(self) -> int:
        return int(self.onsite.shape[-1])

    @property
    def K(self) -> int:
        return int(self.onsite.shape[0])

    @property
    def nl(self) -> int:
        return int(self.lead_l[0].shape[-1])

    @property
    def nr(self) -> int:
        return int(self.lead_r[0].shape[-1])

    @classmethod
    def from_arrays(cls, lead_l: dict, lead_r: dict, onsite, coupling, n_layers: int, vl=None, vr=None,
                    same_leads: bool | None = None) -> "StackedSystem":
        """Upload host arrays (numpy or torch).  ``vl``/``vr`` default to negfpy's
        matched-contact couplings V_L = d10 (or d01^H) and V_R = d01 (core/negf.py:192-201),
        contacting the whole first / last layer."""
        dev = _dev()
        ll = (_c(lead_l["d00"], dev), _c(lead_l["d01"], dev),
              None if lead_l.get("d10") is None else _c(lead_l["d10"], dev))
        if same_leads is None:
            same_leads = lead_r is lead_l
        lr = ll if same_leads else (_c(lead_r["d00"], dev), _c(lead_r["d01"], dev),
                                    None if lead_r.get("d10") is None else _c(lead_r["d10"], dev))
        on = _c(onsite, dev)
        cp = None if coupling is None else _c(coupling, dev)
        n = on.shape[-1]
        if vl is None:
            vl = ll[2] if ll[2] is not None else ll[1].conj().transpose(-1, -2)
            if vl.shape[-2] != n:
                raise ValueError("default left coupling needs the device block order to equal the lead's")
        if vr is None:
            vr = lr[1]
            if vr.shape[-2] != n:
                raise ValueError("default right coupling needs the device block order to equal the lead's")
        return cls(ll, lr, on, cp, int(n_layers), _c(vl, dev), _c(vr, dev), bool(same_leads))

    def transmission(self, omega: torch.Tensor, k_index: torch.Tensor, eta: torch.Tensor,
                     eta_dev: torch.Tensor | None = None, tol: float = 1e-12, maxiter: int = 200,
                     chunk: int | None = None, stream=None, precision: str = "f64") -> dict:
        """T, status and decimation counts for P points (float64/int32 tensors).

        Points are solved in chunks (one decimation and one device-solve
        launch each); by default a chunk is as many points as keep their
        surface GFs within 8 GiB (233,016 points at lead order 48, 58,254 at
        96), at least 4,096.

        ``precision``:
        - "f64": FP64 throughout;
        - "refined": FP64 surface GFs, the device solve from FP32 factors
          refined to FP64 accuracy, FP64 re-solve of the points whose
          refinement fails (``rgf_transmission_refined``); the result also
          carries ``fallback`` (points re-solved in FP64) and ``steps``
          (refinement steps per point);
        - "mixed": FP64 surface GFs, the FP32 sweep without refinement (about
          FP32 accuracy), FP64 re-solve of failed points
          (``rgf_transmission_mixed``)."""
        if precision not in ("f64", "refined", "mixed"):
            raise ValueError(f"unknown precision {precision!r}; expected 'f64', 'refined' or 'mixed'")
        n_fallback = 0
        steps_all = torch.zeros(int(omega.shape[0]), dtype=torch.int32, device=_dev()) \
            if precision == "refined" else None
        dev = _dev()
        P = int(omega.shape[0])
        omega = _r(omega, dev)
        eta = _r(eta, dev)
        eta_dev = eta if eta_dev is None else _r(eta_dev, dev)
        k_index = k_index.to(device=dev, dtype=torch.int32).contiguous()
        T = torch.empty(P, dtype=RDT, device=dev)
        st = torch.empty(P, dtype=torch.int32, device=dev)
        itl = torch.empty(P, dtype=torch.int32, device=dev)
        itr = torch.empty(P, dtype=torch.int32, device=dev)
        if chunk is None:
            per_point = 16 * (self.nl * self.nl + (0 if self.same_leads else self.nr * self.nr))
            chunk = max(4096, (8 << 30) // per_point)
        chunk = max(1, int(chunk))
        for a in range(0, P, chunk):
            b = min(P, a + chunk)
            sl = slice(a, b)
            om, et, ed, ki = omega[sl], eta[sl], eta_dev[sl], k_index[sl]
            rl = sgf_sr(*self.lead_l, om, et, ki, tol, maxiter, stream=stream)
            if self.same_leads:
                rr = rl
                lst = rl["status"]
            else:
                rr = sgf_sr(*self.lead_r, om, et, ki, tol, maxiter, stream=stream)
                lst = torch.where(rl["status"] != 0, rl["status"], rr["status"])
            if precision == "refined":
                t, s, nb, stp = rgf_transmission_refined(self.onsite, self.coupling, self.n_layers, self.vl,
                                                         self.vr, rl["g"], rr["g"], om, ed, ki, lst, stream=stream)
                n_fallback += nb
                steps_all[sl] = stp
            elif precision == "mixed":
                t, s, nb = rgf_transmission_mixed(self.onsite, self.coupling, self.n_layers, self.vl, self.vr,
                                                  rl["g"], rr["g"], om, ed, ki, lst, stream=stream)
                n_fallback += nb
            else:
                t, s = rgf_transmission(self.onsite, self.coupling, self.n_layers, self.vl, self.vr, rl["g"],
                                        rr["g"], om, ed, ki, lst, stream=stream)
            T[sl] = t
            st[sl] = s
            itl[sl] = rl["iters"]
            itr[sl] = rr["iters"]
        return {"T": T, "status": st, "iters_left": itl, "iters_right": itr, "fallback": n_fallback,
                "steps": steps_all}


def cgemm_tf32x3(a: torch.Tensor, b: torch.Tensor, conj_a: bool = False, conj_b: bool = False,
                 stream=None) -> tuple[torch.Tensor, torch.Tensor]:
    """op(a) @ op(b) for batches of complex64 n x n matrices ``[P, n, n]`` on
    tcgen05 tensor cores (3 x TF32 split, ``negf_cgemm_tf32x3``); returns the
    products and a per-product status."""
    lib = _lib.load()
    dev = _dev()
    a = a.to(device=dev, dtype=torch.complex64).contiguous()
    b = b.to(device=dev, dtype=torch.complex64).contiguous()
    P, n, _ = a.shape
    c = torch.empty_like(a)
    st = torch.full((P,), -1, dtype=torch.int32, device=dev)
    _lib.check(lib.negf_cgemm_tf32x3(n, P, _lib.ptr(a), _lib.ptr(b), _lib.ptr(c), int(conj_a), int(conj_b),
                                     _lib.ptr(st), _lib.stream_handle(stream)), "negf_cgemm_tf32x3")
    return c, st


def set_fp32_product_path(n: int, path: int) -> int:
    """Product tiling of the FP32 device sweeps (mixed and refined) at block
    order ``n``: 0 mma.sync warp tiles, 1 tcgen05 128 x n tiles (n <= 128),
    -1 the default.  Process-wide (``negf_set_fp32_product_path``); returns
    the path now in effect."""
    lib = _lib.load()
    rc = lib.negf_set_fp32_product_path(int(n), int(path))
    if rc < 0:
        _lib.check(rc, "negf_set_fp32_product_path")
    return rc
