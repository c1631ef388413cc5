"""CPU oracle for the per-(omega, k) phonon NEGF path.  TEST INFRASTRUCTURE ONLY.

This module restates negfpy's FP64 algorithm for the hot path in plain
NumPy/SciPy, one function per reference routine, each citing the reference
lines it follows (paths relative to the negfpy project root).  It is the
checker for the CUDA path and the timed CPU baseline: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py`` (its ``cpu_baseline`` leg and
``--impl reference`` arm) may import it.  The product package never does.

Parity pin: ``tests/golden/make_golden.py`` runs negfpy itself on the same
seeded inputs and stores its outputs under ``tests/golden/``;
``tests/test_oracle_golden.py`` checks this module against those vectors.

Arithmetic follows the reference exactly where it matters for rounding:
complex128 throughout, Sancho-Rubio products associated left to right as in
``core/surface_gf.py:45-50``, the device system assembled as one sparse
matrix and factored with SuperLU (``core/negf.py:53-69, 229-250, 353``).
"""

from __future__ import annotations

import os

import numpy as np
from scipy import sparse
from scipy.linalg import eig
from scipy.sparse.linalg import splu

HBAR_J_S = 1.054_571_817e-34
KB_J_K = 1.380_649e-23


class OracleError(RuntimeError):
    """Numerical failure, mirroring the reference's RuntimeError cases."""


def sancho_rubio(omega, d00, d01, d10=None, eta=1e-8, tol=1e-12, maxiter=200):
    """Sancho-Rubio decimation, ``core/surface_gf.py:18-81``.

    Returns ``(g_surface, n_iterations)``.  z = (omega + i eta)^2 (``:33``);
    alpha <- d01, beta <- d10 (default d01^H, ``:12-15``), eps = eps_s = d00;
    per sweep g = (z - eps)^-1, eps_s += a g b, eps += a g b + b g a,
    a <- a g a, b <- b g b (``:41-50``); stop when max(|a|, |b|) < tol
    (``:69-76``); non-finite -> error (``:52-66``); maxiter -> error (``:78``).
    """
    z = (omega + 1j * eta) ** 2
    n = d00.shape[0]
    ident = np.eye(n, dtype=np.complex128)
    a = np.array(d01, dtype=np.complex128)
    b = np.array(np.conj(d01).T if d10 is None else d10, dtype=np.complex128)
    e = np.array(d00, dtype=np.complex128)
    es = e.copy()
    for it in range(1, maxiter + 1):
        with np.errstate(over="raise", invalid="raise", divide="raise"):
            try:
                g = np.linalg.inv(z * ident - e)
                agb = a @ g @ b
                bga = b @ g @ a
                es_n = es + agb
                e_n = e + agb + bga
                a_n = a @ g @ a
                b_n = b @ g @ b
            except FloatingPointError as exc:
                raise OracleError("Sancho-Rubio decimation became numerically unstable.") from exc
        if not (np.all(np.isfinite(es_n)) and np.all(np.isfinite(e_n))
                and np.all(np.isfinite(a_n)) and np.all(np.isfinite(b_n))):
            raise OracleError("Sancho-Rubio decimation produced non-finite values.")
        err = max(float(np.max(np.abs(a_n))), float(np.max(np.abs(b_n))))
        es, e, a, b = es_n, e_n, a_n, b_n
        if err < tol:
            return np.linalg.inv(z * ident - es), it
    raise OracleError("Sancho-Rubio decimation did not converge within maxiter.")


def surface_residual(omega, d00, d01, d10=None, eta=1e-8, tol=1e-12, maxiter=200):
    """How well the decimated surface GF solves its own fixed point.

    Runs ``sancho_rubio`` (``core/surface_gf.py:18-81``) and returns
    max|g - (z - d00 - d01 g d10)^-1| / max|g|.  At ordinary points this is
    ~1e-13; near band edges the decimation's cancellations leave it at
    1e-8 ... 1e-5, and there rounding alone moves negfpy's T by about as much.
    """
    g, _ = sancho_rubio(omega, d00, d01, d10, eta, tol, maxiter)
    z = (omega + 1j * eta) ** 2
    d10 = np.conj(d01).T if d10 is None else d10
    n = d00.shape[0]
    fix = np.linalg.inv(z * np.eye(n, dtype=np.complex128) - d00 - d01 @ g @ d10)
    return float(np.max(np.abs(g - fix)) / np.max(np.abs(g)))


def qep_surface_gf(omega, d00, d01, d10=None, eta=1e-8, unit_circle_tol=1e-10):
    """Generalised-eigen (QEP) surface GF, ``core/surface_gf.py:84-133``.

    Independent cross-check of the decimation: linearise
    (c l^2 + a l + b) phi = 0 with a = d00 - z, b = d10, c = d01, keep the n
    modes with |l| < 1, transfer = Phi diag(l) Phi^-1, g = (z - d00 - c T)^-1.
    """
    n = d00.shape[0]
    z = (omega + 1j * eta) ** 2
    ident = np.eye(n, dtype=np.complex128)
    zero = np.zeros((n, n), dtype=np.complex128)
    a = np.asarray(d00, dtype=np.complex128) - z * ident
    b = np.array(np.conj(d01).T if d10 is None else d10, dtype=np.complex128)
    c = np.asarray(d01, dtype=np.complex128)
    lam, vec = eig(np.block([[-a, -b], [ident, zero]]), np.block([[c, zero], [zero, ident]]), right=True)
    ok = np.isfinite(lam)
    lam, vec = lam[ok], vec[:, ok]
    if lam.size < n:
        raise OracleError("QEP surface GF: insufficient finite eigenmodes.")
    mag = np.abs(lam)
    inside = np.where(mag < 1.0 - unit_circle_tol)[0]
    pick = inside[np.argsort(mag[inside])[:n]] if inside.size >= n else np.argsort(mag)[:n]
    phi = vec[n:, pick]
    if np.linalg.matrix_rank(phi) < n:
        raise OracleError("QEP surface GF: rank-deficient mode set.")
    transfer = phi @ np.diag(lam[pick]) @ np.linalg.inv(phi)
    return np.linalg.inv(z * ident - np.asarray(d00, dtype=np.complex128) - c @ transfer)


def self_energy(v, g):
    """Sigma = V g V^H, ``core/negf.py:72-97``."""
    v = np.asarray(v, dtype=np.complex128)
    return v @ g @ np.conj(v).T


def broadening(sigma):
    """Gamma = i (Sigma - Sigma^H), ``core/negf.py:115-116``."""
    return 1j * (sigma - np.conj(sigma).T)


def _assemble_device(onsite, coupling):
    """Block-tridiagonal device matrix, ``core/negf.py:53-69`` (C above, C^H below)."""
    L = len(onsite)
    rows = [[None] * L for _ in range(L)]
    for i in range(L):
        rows[i][i] = sparse.csr_matrix(np.asarray(onsite[i], dtype=np.complex128))
    for i in range(L - 1):
        c = np.asarray(coupling[i], dtype=np.complex128)
        rows[i][i + 1] = sparse.csr_matrix(c)
        rows[i + 1][i] = sparse.csr_matrix(np.conj(c).T)
    if L == 1:
        return sparse.csc_matrix(rows[0][0])
    return sparse.bmat(rows, format="csc", dtype=np.complex128)


def transmission_point(omega, onsite, coupling, lead_l, lead_r, eta=1e-8, eta_device=None,
                       vl=None, vr=None, idx_l=None, idx_r=None, tol=1e-12, maxiter=200,
                       return_parts=False):
    """T(omega) for one k, ``core/negf.py:141-250, 306-357``.

    ``onsite``: L blocks n x n; ``coupling``: L-1 blocks; ``lead_l``/``lead_r``:
    (d00, d01, d10-or-None).  Default couplings: V_L = d10 (or d01^H) and
    V_R = d01 (``:192-201``); default contacts: first n_cL and last n_cR DOFs
    (``:206-227``).  A = (omega + i eta_dev)^2 I - D - Sigma_L - Sigma_R
    (``:245-248``); X = A^-1 E_R by SuperLU, G_LR = X[idx_l] (``:350-354``);
    T = Re Tr[Gamma_L G_LR Gamma_R G_LR^H] (``:356``).
    """
    L = len(onsite)
    n = onsite[0].shape[0]
    dim = L * n
    eta_dev = float(eta if eta_device is None else eta_device)
    d00l, d01l, d10l = lead_l
    d00r, d01r, d10r = lead_r
    if vl is None:
        vl = d10l if d10l is not None else np.conj(d01l).T
    if vr is None:
        vr = d01r
    vl = np.asarray(vl, dtype=np.complex128)
    vr = np.asarray(vr, dtype=np.complex128)
    ncl, ncr = vl.shape[0], vr.shape[0]
    il = np.arange(ncl) if idx_l is None else np.asarray(idx_l, dtype=int).ravel()
    ir = np.arange(dim - ncr, dim) if idx_r is None else np.asarray(idx_r, dtype=int).ravel()
    gl, itl = sancho_rubio(omega, d00l, d01l, d10l, eta, tol, maxiter)
    gr, itr = sancho_rubio(omega, d00r, d01r, d10r, eta, tol, maxiter)
    sl = self_energy(vl, gl)
    sr = self_energy(vr, gr)
    dmat = _assemble_device(onsite, coupling)
    z = (omega + 1j * eta_dev) ** 2
    a = (z * sparse.identity(dim, dtype=np.complex128, format="csc") - dmat).tolil()
    a[np.ix_(il, il)] = a[np.ix_(il, il)] - sl
    a[np.ix_(ir, ir)] = a[np.ix_(ir, ir)] - sr
    rhs = np.zeros((dim, ncr), dtype=np.complex128)
    rhs[ir, :] = np.eye(ncr, dtype=np.complex128)
    x = splu(a.tocsc()).solve(rhs)
    glr = x[il, :]
    t = float(np.real(np.trace(broadening(sl) @ glr @ broadening(sr) @ np.conj(glr).T)))
    if return_parts:
        return t, {"g_l": gl, "g_r": gr, "iters_l": itl, "iters_r": itr, "sigma_l": sl, "sigma_r": sr}
    return t


def lead_surface_dos(omega, d00, d01, d10=None, eta=1e-8, normalize_per_mode=False, tol=1e-12, maxiter=200):
    """DOS = (omega/pi) Re Tr[i (g - g^H)], ``core/dos.py:31-61``."""
    if omega < 0.0:
        raise ValueError("omega must be non-negative.")
    g, _ = sancho_rubio(omega, d00, d01, d10, eta, tol, maxiter)
    dos = float((omega / np.pi) * np.real(np.trace(1j * (g - np.conj(g).T))))
    if normalize_per_mode:
        dos /= d00.shape[0]
    return dos


def thermal_conductance(omega_model, tvals, temperatures, omega_unit_rad_s):
    """kappa(T) = (1/2pi) trapz(kB T(w) x^2 e^-x / (1 - e^-x)^2, w), ``workflows/ifc_bulk.py:408-438``.

    ``omega_model * omega_unit_rad_s`` is omega in rad/s (the reference uses
    its QE unit factor at ``:420``; synthetic blocks are dimensionless, so
    the factor is explicit here).  Small-x series below 1e-6, zero kernel
    at x >= 700.
    """
    w = np.asarray(omega_model, dtype=float) * float(omega_unit_rad_s)
    t = np.asarray(tvals, dtype=float)
    out = np.zeros(len(np.atleast_1d(temperatures)))
    for i, temp in enumerate(np.atleast_1d(np.asarray(temperatures, dtype=float))):
        if temp <= 0.0:
            continue
        x = HBAR_J_S * w / (KB_J_K * temp)
        kern = np.zeros_like(x)
        small = x < 1e-6
        mid = (x >= 1e-6) & (x < 700.0)
        kern[small] = 1.0 - x[small] ** 2 / 12.0
        y = np.exp(-x[mid])
        kern[mid] = x[mid] ** 2 * y / (1.0 - y) ** 2
        f = KB_J_K * t * kern
        out[i] = float(np.sum(0.5 * (f[1:] + f[:-1]) * np.diff(w)) / (2.0 * np.pi))
    return out


# --------------------------------------------------------- workload runs ----
def workload_point_args(wl, wi, ki):
    """Explicit per-point inputs of a ``negfpy_b200.workloads.Workload``."""
    L = wl.n_layers
    on = wl.onsite[ki]
    cp = wl.coupling[ki]
    onsite = [on[0]] * L if on.shape[0] == 1 else list(on)
    coupling = [cp[0]] * (L - 1) if cp.shape[0] == 1 else list(cp)
    ll = (wl.lead_l["d00"][ki], wl.lead_l["d01"][ki], wl.lead_l["d10"][ki])
    lr = (wl.lead_r["d00"][ki], wl.lead_r["d01"][ki], wl.lead_r["d10"][ki])
    vl = None if wl.vl is None else wl.vl[ki]
    vr = None if wl.vr is None else wl.vr[ki]
    return dict(omega=float(wl.omegas[wi]), onsite=onsite, coupling=coupling, lead_l=ll, lead_r=lr,
                eta=wl.eta, eta_device=wl.eta_device, vl=vl, vr=vr,
                idx_l=wl.meta.get("idx_l"), idx_r=wl.meta.get("idx_r"))


_BLAS_VARS = ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS")


def _pool_init():
    for v in _BLAS_VARS:
        os.environ[v] = "1"


def _pool_task(args):
    try:
        return transmission_point(**args)
    except (OracleError, np.linalg.LinAlgError):
        return float("nan")


def _residual_task(args):
    try:
        d00, d01, d10 = args["lead_l"]
        return surface_residual(args["omega"], d00, d01, d10, args["eta"])
    except (OracleError, np.linalg.LinAlgError):
        return float("nan")


def make_pool(processes):
    """Spawn pool with one BLAS thread per worker, as negfpy's process backend
    (``workflows/ifc_bulk.py:1229-1253``, ``:621-670``); spawn, not fork, so it
    is safe to start after CUDA has been initialised."""
    import multiprocessing as mp

    # Children inherit the environment at spawn, before numpy (and its BLAS)
    # is imported in them, so the thread limit must be set here.
    saved = {v: os.environ.get(v) for v in _BLAS_VARS}
    for v in _BLAS_VARS:
        os.environ[v] = "1"
    try:
        return mp.get_context("spawn").Pool(processes, initializer=_pool_init)
    finally:
        for v, old in saved.items():
            if old is None:
                os.environ.pop(v, None)
            else:
                os.environ[v] = old


def transmission_points(wl, pairs, processes=1, pool=None):
    """T for a list of (omega_index, k_index) pairs, serially or on a process pool."""
    args = [workload_point_args(wl, wi, ki) for wi, ki in pairs]
    if pool is None and processes <= 1:
        return np.array([_pool_task(a) for a in args])
    own = pool is None
    if own:
        pool = make_pool(processes)
    try:
        nproc = pool._processes
        return np.array(pool.map(_pool_task, args, chunksize=max(1, len(args) // (4 * nproc))))
    finally:
        if own:
            pool.close()
            pool.join()


def heat_current_from_spectrum(omegas, tvals, temp_left, temp_right):
    """Landauer heat current (W), ``core/thermal_current.py:30-67``: the
    spectral Bose weight kB T_L phi(x_L) - kB T_R phi(x_R), phi(x) = x/expm1(x)
    (series 1 - x/2 + x^2/12 below 1e-6, 0 from 700 on), trapezoid over omega
    in rad/s, divided by 2 pi."""
    hbar, kb = 1.054_571_817e-34, 1.380_649e-23
    om = np.asarray(omegas, dtype=float)

    def phi(x):
        out = np.zeros_like(x)
        small = x < 1e-6
        mid = (x >= 1e-6) & (x < 700.0)
        out[small] = 1.0 - 0.5 * x[small] + x[small] ** 2 / 12.0
        out[mid] = x[mid] / np.expm1(x[mid])
        return out

    w = kb * temp_left * phi(hbar * om / (kb * temp_left)) - kb * temp_right * phi(hbar * om / (kb * temp_right))
    f = w * np.asarray(tvals, dtype=float)
    return float(np.sum(np.diff(om) * (f[1:] + f[:-1]) / 2.0) / (2.0 * np.pi))


def fcs_cumulants(omegas, t1, t2, temp_left, temp_right):
    """(C1, C2) of the heat current, ``core/fcs.py:48-150``: A = kB T phi1(x),
    B = (kB T)^2 phi2(x), phi1 = x/expm1(x) (series 1 - x/2 + x^2/12 - x^4/720
    for |x| < 1e-6), phi2 = x^2 e^x/expm1(x)^2 (series 1 - x^2/12 + x^4/240),
    both 0 from x = 700 on; C1 = trapz(t1 (A_L - A_R))/2pi,
    C2 = trapz(t1 (B_L + B_R) + (t1 + t2) (A_L - A_R)^2)/2pi."""
    hbar, kb = 1.054_571_817e-34, 1.380_649e-23
    om = np.asarray(omegas, dtype=float)

    def phi(x, which):
        out = np.zeros_like(x)
        small = np.abs(x) < 1e-6
        mid = (np.abs(x) >= 1e-6) & (x < 700.0)
        xs = x[small]
        if which == 1:
            out[small] = 1.0 - 0.5 * xs + xs * xs / 12.0 - xs ** 4 / 720.0
            out[mid] = x[mid] / np.expm1(x[mid])
        else:
            out[small] = 1.0 - xs * xs / 12.0 + xs ** 4 / 240.0
            e = np.expm1(x[mid])
            out[mid] = x[mid] ** 2 * (e + 1.0) / (e * e)
        return out

    sl, sr = kb * temp_left, kb * temp_right
    ad = sl * phi(hbar * om / sl, 1) - sr * phi(hbar * om / sr, 1)
    bs = sl * sl * phi(hbar * om / sl, 2) + sr * sr * phi(hbar * om / sr, 2)
    t1, t2 = np.asarray(t1, dtype=float), np.asarray(t2, dtype=float)
    f1 = t1 * ad
    f2 = t1 * bs + (t1 + t2) * ad * ad
    trap = lambda f: float(np.sum(np.diff(om) * (f[1:] + f[:-1]) / 2.0))  # noqa: E731
    return trap(f1) / (2.0 * np.pi), trap(f2) / (2.0 * np.pi)


def device_green_point(omega, onsite, coupling, lead_l, lead_r, eta=1e-8, eta_device=None, vl=None, vr=None,
                       idx_l=None, idx_r=None, tol=1e-12, maxiter=200):
    """(G, Sigma_L, Sigma_R) of the finite device, ``core/negf.py:253-303``:
    the system matrix of ``transmission_point``, G = A^-1 by SuperLU against
    the identity, and the self-energies embedded at the contact indices."""
    L = len(onsite)
    n = onsite[0].shape[0]
    dim = L * n
    eta_dev = float(eta if eta_device is None else eta_device)
    d00l, d01l, d10l = lead_l
    d00r, d01r, d10r = lead_r
    if vl is None:
        vl = d10l if d10l is not None else np.conj(d01l).T
    if vr is None:
        vr = d01r
    vl, vr = np.asarray(vl, dtype=np.complex128), np.asarray(vr, dtype=np.complex128)
    il = np.arange(vl.shape[0]) if idx_l is None else np.asarray(idx_l, dtype=int).ravel()
    ir = np.arange(dim - vr.shape[0], dim) if idx_r is None else np.asarray(idx_r, dtype=int).ravel()
    gl, _ = sancho_rubio(omega, d00l, d01l, d10l, eta, tol, maxiter)
    gr, _ = sancho_rubio(omega, d00r, d01r, d10r, eta, tol, maxiter)
    sl, sr = self_energy(vl, gl), self_energy(vr, gr)
    z = (omega + 1j * eta_dev) ** 2
    a = (z * sparse.identity(dim, dtype=np.complex128, format="csc") - _assemble_device(onsite, coupling)).tolil()
    a[np.ix_(il, il)] = a[np.ix_(il, il)] - sl
    a[np.ix_(ir, ir)] = a[np.ix_(ir, ir)] - sr
    g = splu(a.tocsc()).solve(np.eye(dim, dtype=np.complex128))
    sig_l = np.zeros((dim, dim), dtype=np.complex128)
    sig_r = np.zeros((dim, dim), dtype=np.complex128)
    sig_l[np.ix_(il, il)] = sl
    sig_r[np.ix_(ir, ir)] = sr
    return g, sig_l, sig_r


def surface_residual_points(wl, pairs, pool=None):
    """Left-lead ``surface_residual`` for (omega_index, k_index) pairs of a workload."""
    args = [workload_point_args(wl, wi, ki) for wi, ki in pairs]
    if pool is None:
        return np.array([_residual_task(a) for a in args])
    return np.array(pool.map(_residual_task, args, chunksize=1))
