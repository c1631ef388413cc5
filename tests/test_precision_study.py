"""Why the surface GF stays FP64 (host-only numerics, no GPU).

On the 3D bulk workload (n = 96, eta = 1e-6 omega_max^2) Sancho-Rubio needs
about 20 doubling sweeps at propagating frequencies, and each sweep
alpha <- alpha g alpha doubles the relative error of alpha.  Run in complex64
the decimation therefore loses most of its digits, although the surface GF
itself is well conditioned: rounding only the INPUT blocks to complex64 and
decimating in FP64 moves g by about 1e-6.  The test keeps both facts true on
a propagating point.
"""

from __future__ import annotations

import numpy as np

from negfpy_b200 import workloads as W
from oracle.negf_oracle import sancho_rubio


def _sr_dtype(w, d00, d01, d10, eta, dt, tol, maxiter=200):
    z = (w + 1j * eta) ** 2
    n = d00.shape[0]
    a, b, e, es = d01.astype(dt), d10.astype(dt), d00.astype(dt), d00.astype(dt)
    eye = np.eye(n, dtype=dt)
    for _ in range(maxiter):
        g = np.linalg.inv(z * eye - e).astype(dt)
        ag, bg = a @ g, b @ g
        agb, bga = ag @ b, bg @ a
        es, e = es + agb, e + agb + bga
        a, b = ag @ a, bg @ b
        if max(np.abs(a).max(), np.abs(b).max()) < tol:
            break
    return np.linalg.inv(z * np.eye(n) - es.astype(np.complex128))


def test_complex64_decimation_is_unstable_but_the_problem_is_not():
    wl = W.bulk_workload()
    wi, ki = 2489, 243  # a propagating point (20 decimation sweeps in FP64)
    w = wl.omegas[wi]
    d00, d01, d10 = (wl.lead_l[x][ki] for x in ("d00", "d01", "d10"))
    g64, it = sancho_rubio(w, d00, d01, d10, wl.eta, 1e-12, 200)
    assert it >= 18
    rel = lambda g: float(np.abs(g - g64).max() / np.abs(g64).max())  # noqa: E731
    g_in32 = sancho_rubio(w, *(x.astype(np.complex64).astype(np.complex128) for x in (d00, d01, d10)), wl.eta,
                          1e-12, 200)[0]
    assert rel(g_in32) < 1e-5
    g32 = _sr_dtype(w, d00, d01, d10, wl.eta, np.complex64, 1e-6)
    assert rel(g32) > 1e-4
