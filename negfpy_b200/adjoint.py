"""Hand-written adjoint of T(omega, k) and kappa(T) with respect to device force constants.

negfpy has no derivatives; this extends its path (``core/negf.py:306-357``,
the device solve, and ``workflows/ifc_bulk.py:408-438``, kappa).  For a device
whose k-space blocks depend linearly on parameters theta
(``hetero.HeteroModel``: spring constants around an interface), with
A = (omega + i eta)^2 I - D(theta) - Sigma_L - Sigma_R and G = A^-1,

    dT = 2 Re sum_ij Tr[dD_ij X_ji],  X_ji = G_{j,L-1} Gamma_R G_{0,L-1}^H Gamma_L G_{0,i}.

``negf_rgf_adjoint_f64`` accumulates sum_p w_p X per k for weights w (the
incoming gradient of T); torch's gradient of the blocks is then 2 conj(X^T),
and torch autograd carries it through the block builder to the spring
constants and masses.
The adjoint kernel recomputes the forward sweeps (nothing but theta is kept
between forward and backward: checkpointing by recomputation).  The leads do
not depend on theta, so their surface Green's functions are computed once per
problem and reused by every forward and backward call.

``TransmissionFunction`` is the autograd primitive (blocks -> T[W, K]);
``kappa`` composes it with a block builder, the k mean and the Bose-weighted
trapezoid in torch.
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


class DeviceSolve:
    """The theta-independent part of a differentiable solve: points, lead surface
    GFs and contact couplings of a layer-resolved device between two leads."""

    def __init__(self, lead_l: dict, lead_r: dict, vl, vr, n_layers: int, omegas, n_k: int, eta: float,
                 tol: float = 1e-12, maxiter: int = 200):
        dev = _lib.require_cuda()
        c = engine._c
        self.om = torch.as_tensor(np.asarray(omegas, float), device=dev)
        self.W, self.K, self.L = self.om.numel(), int(n_k), int(n_layers)
        wi = torch.arange(self.W, device=dev).repeat_interleave(self.K)
        self.ki = torch.arange(self.K, device=dev, dtype=torch.int32).repeat(self.W)
        self.omega = self.om[wi].contiguous()
        self.eta = torch.full_like(self.omega, eta)
        rl = engine.sgf_sr(c(lead_l["d00"]), c(lead_l["d01"]), c(lead_l["d10"]), self.omega, self.eta, self.ki, tol,
                           maxiter)
        rr = engine.sgf_sr(c(lead_r["d00"]), c(lead_r["d01"]), c(lead_r["d10"]), self.omega, self.eta, self.ki, tol,
                           maxiter)
        self.g_l, self.g_r = rl["g"], rr["g"]
        self.lead_status = torch.where(rl["status"] != 0, rl["status"], rr["status"]).contiguous()
        self.vl, self.vr = c(vl), c(vr)

    def _check(self, st: torch.Tensor) -> None:
        bad = int((st != 0).sum())
        if bad:
            raise RuntimeError(f"device solve failed at {bad} of {st.numel()} (omega, k) points")

    def transmission(self, onsite: torch.Tensor, coupling: torch.Tensor) -> torch.Tensor:
        """T[W, K] for layer-resolved blocks onsite [K, L, n, n], coupling [K, L-1, n, n]."""
        T, st = engine.rgf_transmission(onsite.contiguous(), coupling.contiguous(), self.L, self.vl, self.vr, self.g_l,
                                        self.g_r, self.omega, self.eta, self.ki, self.lead_status)
        self._check(st)
        return T.reshape(self.W, self.K)

    def vjp(self, onsite: torch.Tensor, coupling: torch.Tensor, weight: torch.Tensor):
        """(T[W, K], X_onsite, X_coupling) with sum_p weight[p] dT_p = 2 Re sum Tr[dD X]
        over the adjoint blocks, in one launch of the adjoint kernel."""
        w = weight.reshape(-1).to(device=self.omega.device, dtype=torch.float64).contiguous()
        T, st, g_on, g_cp = engine.rgf_adjoint(onsite.contiguous(), coupling.contiguous(), self.L, self.vl, self.vr,
                                               self.g_l, self.g_r, self.omega, self.eta, self.ki, self.lead_status, w)
        self._check(st)
        return T.reshape(self.W, self.K), g_on, g_cp


def block_grads(x_onsite: torch.Tensor, x_coupling: torch.Tensor):
    """torch's gradient of a real loss with respect to complex blocks D, given
    dLoss = 2 Re Tr[dD X] per block: 2 conj(X^T) elementwise."""
    return 2.0 * x_onsite.conj().transpose(-1, -2), 2.0 * x_coupling.conj().transpose(-1, -2)


class TransmissionFunction(torch.autograd.Function):
    """T[W, K] = TransmissionFunction.apply(onsite, coupling, solve) for
    layer-resolved complex blocks.  The backward takes the incoming gradient of
    T as the adjoint weights, runs the adjoint kernel (which recomputes the
    forward sweeps) and returns the gradients of the blocks, so that any
    torch-differentiable block builder carries them on to its parameters."""

    @staticmethod
    def forward(ctx, onsite: torch.Tensor, coupling: torch.Tensor, solve: DeviceSolve) -> torch.Tensor:
        ctx.solve = solve
        ctx.save_for_backward(onsite.detach(), coupling.detach())
        return solve.transmission(onsite.detach(), coupling.detach())

    @staticmethod
    def backward(ctx, grad_t):
        on, cp = ctx.saved_tensors
        _, x_on, x_cp = ctx.solve.vjp(on, cp, grad_t)
        g_on, g_cp = block_grads(x_on, x_cp)
        return g_on, g_cp, None


class HeteroKappaProblem(DeviceSolve):
    """kappa(theta, masses) of a ``HeteroModel`` between its leads A and B on an (omega x k) grid."""

    def __init__(self, model: HeteroModel, kpoints, omegas, eta: float, temperature: float = 300.0,
                 omega_unit_rad_s: float = 1.0, tol: float = 1e-12, maxiter: int = 200,
                 w_kappa: torch.Tensor | None = None):
        """``w_kappa``: kappa weights of these omegas when they are a shard of a
        larger grid (default: the trapezoid over these omegas alone)."""
        self.model, self.kpoints = model, list(kpoints)
        self.eta0, self.temperature, self.omega_unit_rad_s = float(eta), float(temperature), float(omega_unit_rad_s)
        la = model.lead_blocks("A", self.kpoints)
        lb = model.lead_blocks("B", self.kpoints)
        vl = np.zeros((len(self.kpoints), model.n, model.n_a), dtype=complex)
        vl[:, model.contact_left_indices(), :] = la["d10"]
        super().__init__(la, lb, vl, lb["d01"], model.L, omegas, len(self.kpoints), eta, tol, maxiter)
        self.w_kappa = (kappa_weights(self.om, temperature, omega_unit_rad_s) if w_kappa is None
                        else torch.as_tensor(w_kappa, dtype=torch.float64, device=self.om.device))

    def blocks(self, theta: torch.Tensor, masses: torch.Tensor | None = None):
        return self.model.blocks(theta, self.kpoints, masses)

    def kappa_of_t(self, T: torch.Tensor) -> torch.Tensor:
        return (self.w_kappa * T.mean(dim=1)).sum()

    def transmission_theta(self, theta: torch.Tensor, masses: torch.Tensor | None = None) -> torch.Tensor:
        on, cp = self.blocks(theta.detach(), None if masses is None else masses.detach())
        return self.transmission(on, cp)

    def kappa_and_grad(self, theta: torch.Tensor, masses: torch.Tensor | None = None):
        """(kappa, dkappa/dtheta, dkappa/dmasses) with one adjoint launch: the
        weights dkappa/dT are known before the solve, so no separate forward
        solve is needed; torch autograd carries the block gradients through
        the block builder."""
        th = theta.detach().clone().requires_grad_(True)
        m0 = torch.as_tensor(self.model.mass, device=th.device) if masses is None else masses
        m = m0.detach().clone().to(dtype=torch.float64).requires_grad_(True)
        on, cp = self.blocks(th, m)
        w = (self.w_kappa[:, None] / self.K).expand(self.W, self.K)
        T, x_on, x_cp = self.vjp(on.detach(), cp.detach(), w)
        g_on, g_cp = block_grads(x_on, x_cp)
        dth, dm = torch.autograd.grad([on, cp], [th, m], [g_on, g_cp])
        return self.kappa_of_t(T), dth, dm


def kappa(theta: torch.Tensor, problem: HeteroKappaProblem, masses: torch.Tensor | None = None) -> torch.Tensor:
    """kappa(T) in W/K, differentiable in theta (and masses) through ``TransmissionFunction``."""
    on, cp = problem.blocks(theta, masses)
    return problem.kappa_of_t(TransmissionFunction.apply(on, cp, problem))


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
