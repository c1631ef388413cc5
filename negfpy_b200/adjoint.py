"""Hand-written adjoint of T(omega, k) and kappa(T) with respect to device force constants.

negfpy has no derivatives; this extends its path (``core/negf.py:306-357``,
the device solve, and ``workflows/ifc_bulk.py:408-438``, kappa).  For a device
whose k-space blocks depend linearly on parameters theta
(``hetero.HeteroModel``: spring constants around an interface), with
A = (omega + i eta)^2 I - D(theta) - Sigma_L - Sigma_R and G = A^-1,

    dT = 2 Re sum_ij Tr[dD_ij X_ji],  X_ji = G_{j,L-1} Gamma_R G_{0,L-1}^H Gamma_L G_{0,i}.

``negf_rgf_adjoint_f64`` accumulates sum_p w_p X per k for weights w (the
incoming gradient of T), ``HeteroModel.contract`` maps the blocks onto theta.
The adjoint kernel recomputes the forward sweeps (nothing but theta is kept
between forward and backward: checkpointing by recomputation).  The leads do
not depend on theta, so their surface Green's functions are computed once per
problem and reused by every forward and backward call.

``TransmissionFunction`` is the autograd primitive (theta -> T[W, K]);
``kappa`` composes it with the k mean and the Bose-weighted trapezoid in torch.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib, engine
from .hetero import HeteroModel

HBAR_J_S = 1.054_571_817e-34
KB_J_K = 1.380_649e-23


def kappa_weights(omegas: torch.Tensor, temperature: float, omega_unit_rad_s: float) -> torch.Tensor:
    """w[w] with kappa = sum_w w[w] Tbar[w]: trapezoid over omega of
    Tbar * hbar omega dn/dT / (2 pi) in W/K, as ``_thermal_conductance_from_spectrum``
    (``workflows/ifc_bulk.py:408-438``) with omega in model units times
    ``omega_unit_rad_s``."""
    wr = omegas.to(torch.float64) * omega_unit_rad_s
    x = HBAR_J_S * wr / (KB_J_K * temperature)
    ker = torch.zeros_like(x)
    small = x < 1e-6
    mid = (x >= 1e-6) & (x < 700.0)
    ker[small] = 1.0 - x[small] ** 2 / 12.0
    y = torch.exp(-x[mid])
    ker[mid] = x[mid] ** 2 * y / (1.0 - y) ** 2
    dw = torch.diff(wr)
    trap = torch.zeros_like(wr)
    trap[:-1] += 0.5 * dw
    trap[1:] += 0.5 * dw
    return trap * KB_J_K * ker / (2.0 * np.pi)


class HeteroKappaProblem:
    """T(theta) on an (omega x k) grid for a ``HeteroModel`` between its leads A and B."""

    def __init__(self, model: HeteroModel, kpoints, omegas, eta: float, temperature: float = 300.0,
                 omega_unit_rad_s: float = 1.0, tol: float = 1e-12, maxiter: int = 200):
        dev = _lib.require_cuda()
        self.model, self.kpoints = model, list(kpoints)
        self.om = torch.as_tensor(np.asarray(omegas, float), device=dev)
        W, K = self.om.numel(), len(self.kpoints)
        self.W, self.K = W, K
        wi = torch.arange(W, device=dev).repeat_interleave(K)
        self.ki = torch.arange(K, device=dev, dtype=torch.int32).repeat(W)
        self.omega = self.om[wi].contiguous()
        self.eta = torch.full_like(self.omega, eta)
        la = model.lead_blocks("A", self.kpoints)
        lb = model.lead_blocks("B", self.kpoints)
        c = engine._c
        rl = engine.sgf_sr(c(la["d00"]), c(la["d01"]), c(la["d10"]), self.omega, self.eta, self.ki, tol, maxiter)
        rr = engine.sgf_sr(c(lb["d00"]), c(lb["d01"]), c(lb["d10"]), self.omega, self.eta, self.ki, tol, maxiter)
        self.g_l, self.g_r = rl["g"], rr["g"]
        self.lead_status = torch.where(rl["status"] != 0, rl["status"], rr["status"]).contiguous()
        vl = np.zeros((K, model.n, model.n_a), dtype=complex)
        vl[:, model.contact_left_indices(), :] = la["d10"]
        self.vl = c(vl)
        self.vr = c(lb["d01"])
        self.w_kappa = kappa_weights(self.om, temperature, omega_unit_rad_s)

    def _check(self, st: torch.Tensor) -> None:
        bad = int((st != 0).sum())
        if bad:
            raise RuntimeError(f"device solve failed at {bad} of {st.numel()} (omega, k) points")

    def transmission(self, theta: torch.Tensor) -> torch.Tensor:
        """T[W, K] (float64) for spring values theta."""
        on, cp = self.model.blocks(theta.detach(), self.kpoints)
        T, st = engine.rgf_transmission(on.contiguous(), cp.contiguous(), self.model.L, self.vl, self.vr, self.g_l,
                                        self.g_r, self.omega, self.eta, self.ki, self.lead_status)
        self._check(st)
        return T.reshape(self.W, self.K)

    def vjp(self, theta: torch.Tensor, weight: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
        """(T[W, K], sum_p weight[p] dT_p/dtheta) in one adjoint launch."""
        on, cp = self.model.blocks(theta.detach(), self.kpoints)
        w = weight.reshape(-1).to(device=self.omega.device, dtype=torch.float64).contiguous()
        T, st, g_on, g_cp = engine.rgf_adjoint(on.contiguous(), cp.contiguous(), self.model.L, self.vl, self.vr,
                                               self.g_l, self.g_r, self.omega, self.eta, self.ki, self.lead_status, w)
        self._check(st)
        return T.reshape(self.W, self.K), self.model.contract(g_on, g_cp, self.kpoints)

    def kappa_of_t(self, T: torch.Tensor) -> torch.Tensor:
        return (self.w_kappa * T.mean(dim=1)).sum()

    def kappa_and_grad(self, theta: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
        """kappa and dkappa/dtheta with the adjoint weights w_p = dkappa/dT_p."""
        w = (self.w_kappa[:, None] / self.K).expand(self.W, self.K)
        T, g = self.vjp(theta, w)
        return self.kappa_of_t(T), g


class TransmissionFunction(torch.autograd.Function):
    """T[W, K] = TransmissionFunction.apply(theta, problem).  The backward
    takes the incoming gradient of T as the adjoint weights, recomputes the
    forward sweeps in the adjoint kernel and returns grad_theta."""

    @staticmethod
    def forward(ctx, theta: torch.Tensor, problem: HeteroKappaProblem) -> torch.Tensor:
        ctx.problem = problem
        ctx.save_for_backward(theta.detach())
        return problem.transmission(theta)

    @staticmethod
    def backward(ctx, grad_t):
        (theta,) = ctx.saved_tensors
        _, g = ctx.problem.vjp(theta, grad_t)
        return g, None


def kappa(theta: torch.Tensor, problem: HeteroKappaProblem) -> torch.Tensor:
    """kappa(T) in W/K, differentiable in theta through ``TransmissionFunction``."""
    return problem.kappa_of_t(TransmissionFunction.apply(theta, problem))


def hetero_problem(model: HeteroModel | None = None, n_k: int = 8, n_omega: int = 256, eta_rel: float = 1e-6,
                   temperature: float = 300.0) -> HeteroKappaProblem:
    """The heterojunction problem: lead A (order 48) | 30 layers | lead B (order
    72), ky on a midpoint grid of n_k points, n_omega midpoints up to 1.05
    omega_max of the two leads, eta = eta_rel omega_max^2, omega_max mapped to
    2 pi 15 THz for kappa."""
    from .workloads import kline, omega_unit_for

    model = model or HeteroModel()
    kpoints = [(float(k),) for k in kline(n_k)]
    wmax = model.omega_max()
    om = (np.arange(n_omega) + 0.5) * (1.05 * wmax / n_omega)
    return HeteroKappaProblem(model, kpoints, om, eta_rel * wmax * wmax, temperature, omega_unit_for(wmax))
