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

# Adjoint blocks of each point stored separately and summed per k in a fixed
# order (negf_rgf_adjoint_points_f64 / negf_sgf_adjoint_points_f64), so that
# kappa's gradient is the same bit for bit from run to run; False adds them
# with FP64 atomics instead (rounding-level run-to-run differences).
DETERMINISTIC = True

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
                                               self.g_l, self.g_r, self.omega, self.eta, self.ki, self.lead_status, w,
                                               deterministic=DETERMINISTIC)
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


    # ----------------------------------------------- leads as variables too
    def leads(self, masses: torch.Tensor | None = None, phi_a: torch.Tensor | None = None,
              phi_b: torch.Tensor | None = None):
        """Lead blocks and contact couplings as torch tensors of the current
        parameters: (lead A, lead B, V_L [K, n, n_A], V_R [K, n, n_B]);
        V_L holds lead A's d10 on the device rows of layer 0 and V_R is lead
        B's d01, the couplings ``__init__`` builds from the fixed leads."""
        dev = self.om.device
        mdl = self.model
        la = mdl.lead_blocks_torch("A", self.kpoints, phi_a, masses, device=dev)
        lb = mdl.lead_blocks_torch("B", self.kpoints, phi_b, masses, device=dev)
        rows = torch.as_tensor(mdl.contact_left_indices(), device=dev)
        vl = torch.zeros((self.K, mdl.n, mdl.n_a), dtype=torch.complex128, device=dev)
        vl = vl.index_copy(1, rows, la["d10"])
        return la, lb, vl, lb["d01"]

    def _points(self):
        return PointGrid(self.omega, self.eta, self.ki, self.W, self.K, self.L)

    def kappa_full(self, theta: torch.Tensor, masses: torch.Tensor | None = None, phi_a: torch.Tensor | None = None,
                   phi_b: torch.Tensor | None = None) -> float:
        """kappa with every part rebuilt from the parameters: both leads'
        blocks and surface GFs (decimated again), the couplings and the
        device (the forward of ``kappa_and_grad_all``)."""
        with torch.no_grad():
            on, cp = self.model.blocks(theta, self.kpoints, masses, phi_a=phi_a, phi_b=phi_b)
            la, lb, vl, vr = self.leads(masses, phi_a, phi_b)
            T = transport(on, cp, vl, vr, la["d00"], la["d01"], lb["d00"], lb["d01"], self._points(), grad=False)[0]
        return float(self.kappa_of_t(T))

    def kappa_and_grad_all(self, theta: torch.Tensor, masses: torch.Tensor | None = None,
                           phi_a: torch.Tensor | None = None, phi_b: torch.Tensor | None = None):
        """(kappa, dkappa/dtheta, dkappa/dmasses, dkappa/dphi_a, dkappa/dphi_b)
        with the leads differentiated too: both decimations, one device
        adjoint launch that also returns the contact self-energy adjoints, one
        surface-GF adjoint launch per lead, then one autograd pass through the
        device and lead block builders."""
        dev = self.om.device
        mdl = self.model

        def leaf(x, default):
            x = torch.as_tensor(default, device=dev) if x is None else x
            return x.detach().clone().to(device=dev, dtype=torch.float64).requires_grad_(True)

        th = leaf(theta, mdl.theta0)
        m = leaf(masses, mdl.mass)
        pa = leaf(phi_a, mdl.phi0_a)
        pb = leaf(phi_b, mdl.phi0_b)
        on, cp = mdl.blocks(th, self.kpoints, m, phi_a=pa, phi_b=pb)
        la, lb, vl, vr = self.leads(m, pa, pb)
        w = (self.w_kappa[:, None] / self.K).expand(self.W, self.K)
        T, grads = transport_vjp(on, cp, vl, vr, la["d00"], la["d01"], lb["d00"], lb["d01"], self._points(), w)
        outs = [on, cp, vl, vr, la["d00"], la["d01"], lb["d00"], lb["d01"]]
        d = torch.autograd.grad(outs, [th, m, pa, pb], list(grads), allow_unused=True)
        d = [torch.zeros_like(x) if g is None else g for g, x in zip(d, (th, m, pa, pb))]
        return (self.kappa_of_t(T), *d)


class PointGrid:
    """The (omega, k) points of a solve: omega-major, ``W`` x ``K``, device of ``L`` layers."""

    def __init__(self, omega, eta, ki, W, K, L):
        self.omega, self.eta, self.ki, self.W, self.K, self.L = omega, eta, ki, W, K, L


def _x_to_grad(x: torch.Tensor) -> torch.Tensor:
    """torch's gradient of a real loss from its adjoint X in dLoss = 2 Re Tr[dY X]: 2 conj(X^T)."""
    return 2.0 * x.conj().transpose(-1, -2)


def transport(onsite, coupling, vl, vr, l_d00, l_d01, r_d00, r_d01, pts: PointGrid, grad: bool = False,
              tol: float = 1e-12, maxiter: int = 200):
    """T[W, K] of a layer-resolved device between two leads given as blocks
    (d10 = d01^H): decimation of both leads, then the device solve.  Returns
    (T, (g_l, g_r, lead_status))."""
    g_l, g_r, lst = _decimate(l_d00, l_d01, r_d00, r_d01, pts, tol, maxiter)
    T, st = engine.rgf_transmission(onsite.detach().contiguous(), coupling.detach().contiguous(), pts.L,
                                    vl.detach().contiguous(), vr.detach().contiguous(), g_l, g_r, pts.omega,
                                    pts.eta, pts.ki, lst)
    bad = int((st != 0).sum())
    if bad:
        raise RuntimeError(f"device solve failed at {bad} of {st.numel()} (omega, k) points")
    return T.reshape(pts.W, pts.K), (g_l, g_r, lst)


def transport_vjp(onsite, coupling, vl, vr, l_d00, l_d01, r_d00, r_d01, pts: PointGrid, weight: torch.Tensor,
                  g=None, tol: float = 1e-12, maxiter: int = 200):
    """(T[W, K], torch gradients of sum weight*T with respect to onsite,
    coupling, vl, vr, l_d00, l_d01, r_d00, r_d01).  The surface GFs ``g`` =
    (g_l, g_r, lead_status) are decimated here unless given; the device
    adjoint recomputes its sweeps and returns the contact self-energy
    adjoints, which the surface-GF adjoint kernel turns into lead-block and
    coupling gradients (the d10 = d01^H part folded into d01)."""
    if g is None:
        g = _decimate(l_d00, l_d01, r_d00, r_d01, pts, tol, maxiter)
    g_l, g_r, lst = g
    w = weight.reshape(-1).to(device=pts.omega.device, dtype=torch.float64).contiguous()
    T, st, x_on, x_cp, xs_l, xs_r = engine.rgf_adjoint(onsite.detach().contiguous(), coupling.detach().contiguous(),
                                                       pts.L, vl.detach().contiguous(), vr.detach().contiguous(),
                                                       g_l, g_r, pts.omega, pts.eta, pts.ki, lst, w, want_sigma=True,
                                                       deterministic=DETERMINISTIC)
    bad = int((st != 0).sum())
    if bad:
        raise RuntimeError(f"device solve failed at {bad} of {st.numel()} (omega, k) points")
    al = engine.sgf_adjoint(l_d01.detach(), None, vl.detach(), g_l, xs_l, pts.ki, lst, tol, maxiter,
                            deterministic=DETERMINISTIC)
    ar = engine.sgf_adjoint(r_d01.detach(), None, vr.detach(), g_r, xs_r, pts.ki, lst, tol, maxiter,
                            deterministic=DETERMINISTIC)
    for a in (al, ar):
        nb = int((a["status"] != 0).sum())
        if nb:
            raise RuntimeError(f"surface-GF adjoint failed at {nb} of {a['status'].numel()} points")
    grads = (_x_to_grad(x_on), _x_to_grad(x_cp), _x_to_grad(al["v"]), _x_to_grad(ar["v"]), _x_to_grad(al["h00"]),
             _x_to_grad(al["h01"]), _x_to_grad(ar["h00"]), _x_to_grad(ar["h01"]))
    return T.reshape(pts.W, pts.K), grads


def _decimate(l_d00, l_d01, r_d00, r_d01, pts, tol, maxiter):
    rl = engine.sgf_sr(l_d00.detach().contiguous(), l_d01.detach().contiguous(), None, pts.omega, pts.eta, pts.ki,
                       tol, maxiter)
    rr = engine.sgf_sr(r_d00.detach().contiguous(), r_d01.detach().contiguous(), None, pts.omega, pts.eta, pts.ki,
                       tol, maxiter)
    return rl["g"], rr["g"], torch.where(rl["status"] != 0, rl["status"], rr["status"]).contiguous()


class TransportFunction(torch.autograd.Function):
    """T[W, K] = TransportFunction.apply(onsite, coupling, vl, vr, l_d00,
    l_d01, r_d00, r_d01, points): the whole solve -- both leads decimated from
    their blocks (d10 = d01^H), the device between them -- differentiable in
    every block.  The forward keeps the surface GFs (one n x n matrix per
    point and lead); the backward recomputes the device sweeps inside the
    adjoint kernel and differentiates the surface GFs implicitly through
    their fixed point."""

    @staticmethod
    def forward(ctx, onsite, coupling, vl, vr, l_d00, l_d01, r_d00, r_d01, pts: PointGrid):
        T, g = transport(onsite, coupling, vl, vr, l_d00, l_d01, r_d00, r_d01, pts)
        ctx.pts, ctx.g = pts, g
        ctx.save_for_backward(onsite.detach(), coupling.detach(), vl.detach(), vr.detach(), l_d00.detach(),
                              l_d01.detach(), r_d00.detach(), r_d01.detach())
        return T

    @staticmethod
    def backward(ctx, grad_t):
        blocks = ctx.saved_tensors
        _, grads = transport_vjp(*blocks, ctx.pts, grad_t, g=ctx.g)
        return (*grads, None)


def kappa_all(theta: torch.Tensor, problem: HeteroKappaProblem, masses: torch.Tensor | None = None,
              phi_a: torch.Tensor | None = None, phi_b: torch.Tensor | None = None) -> torch.Tensor:
    """kappa in W/K through ``TransportFunction``: differentiable in theta, the
    masses and the two material tables, leads included."""
    on, cp = problem.model.blocks(theta, problem.kpoints, masses, phi_a=phi_a, phi_b=phi_b)
    la, lb, vl, vr = problem.leads(masses, phi_a, phi_b)
    T = TransportFunction.apply(on, cp, vl, vr, la["d00"], la["d01"], lb["d00"], lb["d01"], problem._points())
    return problem.kappa_of_t(T)


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
