"""Drop-in ``surface_gf`` API (negfpy ``core/surface_gf.py``) on the GPU.

Only Sancho-Rubio decimation runs here, on the CUDA kernel
``negf_sgf_sr_f64``.  The eigenmode (QEP) methods are negfpy's CPU
cross-check for decimation; they are not part of the GPU path and raise
``NotImplementedError`` rather than silently running on the host.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib, engine

SR_NAMES = {"sancho_rubio", "sancho-rubio", "sr"}
QEP_NAMES = {
    "generalized_eigen", "generalized-eigen", "eig", "gep",
    "generalized_eigen_svd", "generalized-eigen-svd", "ge_svd", "gep_svd",
    "legacy_eigen_svd", "legacy-eigen-svd", "legacy", "old_svd",
}

# Messages of the reference's RuntimeError cases (core/surface_gf.py:52-79).
MSG_NONFINITE = ("Sancho-Rubio decimation produced non-finite values. "
                 "Try a larger eta or a different surface_gf method.")
MSG_MAXITER = "Sancho-Rubio decimation did not converge within maxiter."
MSG_UNSTABLE = ("Sancho-Rubio decimation became numerically unstable. "
                "Try a larger eta or a different surface_gf method.")


def check_method(method: str) -> None:
    """Validate a surface-GF method name exactly as negfpy's dispatcher (``:254-311``)."""
    m = method.strip().lower()
    if m in SR_NAMES:
        return
    if m in QEP_NAMES:
        raise NotImplementedError(
            f"surface_gf method '{method}' is an eigenmode (QEP) solver, which serves as the CPU oracle for "
            "decimation and is not part of the GPU path; use method='sancho_rubio'.")
    raise ValueError(
        "Unknown surface GF method. Use one of: "
        "'sancho_rubio', 'generalized_eigen', 'generalized_eigen_svd', 'legacy_eigen_svd'.")


def raise_for_status(status: int) -> None:
    """Map a kernel status to the exception negfpy raises for the same failure."""
    if status == _lib.OK:
        return
    if status == _lib.MAXITER:
        raise RuntimeError(MSG_MAXITER)
    if status == _lib.NONFINITE:
        raise RuntimeError(MSG_NONFINITE)
    if status == _lib.UNSTABLE:
        raise RuntimeError(MSG_UNSTABLE)
    if status == _lib.SINGULAR:
        raise np.linalg.LinAlgError("Singular matrix")
    raise RuntimeError(f"NEGF kernel failed with status {status}")


def surface_gf_sancho_rubio(omega: float, d00, d01, d10=None, eta: float = 1e-8, tol: float = 1e-12,
                            maxiter: int = 200) -> np.ndarray:
    """Retarded surface Green's function of a semi-infinite lead (negfpy ``:18-81``)."""
    d00 = np.asarray(d00)
    d01 = np.asarray(d01)
    if d00.ndim != 2 or d00.shape[0] != d00.shape[1] or d01.shape != d00.shape:
        raise ValueError("d00 and d01 must be square matrices of the same shape.")
    if d10 is not None and np.shape(d10) != d00.shape:
        raise ValueError("d10 must have the same shape as d00.")
    dev = _lib.require_cuda()
    om = torch.tensor([float(omega)], dtype=torch.float64, device=dev)
    et = torch.tensor([float(eta)], dtype=torch.float64, device=dev)
    r = engine.sgf_sr(engine._c(d00), engine._c(d01), None if d10 is None else engine._c(d10), om, et,
                      None, tol, maxiter)
    raise_for_status(int(r["status"].item()))
    return r["g"][0].cpu().numpy()


def surface_gf(omega: float, d00, d01, d10=None, eta: float = 1e-8, *, method: str = "sancho_rubio",
               tol: float = 1e-12, maxiter: int = 200, unit_circle_tol: float = 1e-10,
               svd_rcond: float = 1e-12) -> np.ndarray:
    """Surface GF with negfpy's dispatcher signature (``core/surface_gf.py:254-311``)."""
    check_method(method)
    return surface_gf_sancho_rubio(omega, d00, d01, d10, eta=eta, tol=tol, maxiter=maxiter)


def _qep_unavailable(*_a, **_k):
    check_method("generalized_eigen")


surface_gf_generalized_eigen = _qep_unavailable
surface_gf_generalized_eigen_svd = _qep_unavailable
surface_gf_legacy_eigen_svd = _qep_unavailable
