"""Adjoint of the device solve: dkappa/dtheta and T vector-Jacobian products.

Checked three ways: against torch autograd through a dense solve of the whole
device matrix (block order n = 24, the same lead surface GFs), against central
finite differences (h = 1e-6) of the forward kernels on 50 random parameters
of the heterojunction (lead 48 | 30 layers of order 72 | lead 72, 2000
parameters), and T of the heterojunction against the oracle.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from negfpy_b200 import adjoint  # noqa: E402
from negfpy_b200.hetero import HeteroModel  # noqa: E402


def dense_transmission(problem, theta):
    """T[W, K] by a dense solve of A = (w + i eta)^2 - D - Sigma over all layers (torch, differentiable)."""
    m = problem.model
    on, cp = m.blocks(theta, problem.kpoints)
    K, L, n = on.shape[0], m.L, m.n
    N = L * n
    D = torch.zeros((K, N, N), dtype=torch.complex128, device=on.device)
    for l in range(L):
        D[:, l * n:(l + 1) * n, l * n:(l + 1) * n] = on[:, l]
    for l in range(L - 1):
        D[:, l * n:(l + 1) * n, (l + 1) * n:(l + 2) * n] = cp[:, l]
        D[:, (l + 1) * n:(l + 2) * n, l * n:(l + 1) * n] = cp[:, l].conj().transpose(-1, -2)
    ki = problem.ki.long()
    vl, vr = problem.vl[ki], problem.vr[ki]
    sl = vl @ problem.g_l @ vl.conj().transpose(-1, -2)
    sr = vr @ problem.g_r @ vr.conj().transpose(-1, -2)
    z = (problem.omega + 1j * problem.eta) ** 2
    eye = torch.eye(N, dtype=torch.complex128, device=on.device)
    A = z[:, None, None] * eye - D[ki]
    pad_l = torch.zeros_like(A)
    pad_l[:, :n, :n] = sl
    pad_l[:, N - n:, N - n:] = sr
    A = A - pad_l
    rhs = eye[:, N - n:].expand(A.shape[0], N, n)
    g = torch.linalg.solve(A, rhs)[:, :n, :]
    gam_l = 1j * (sl - sl.conj().transpose(-1, -2))
    gam_r = 1j * (sr - sr.conj().transpose(-1, -2))
    t = torch.einsum("pab,pbc,pcd,pad->p", gam_l, g, gam_r, g.conj()).real
    return t.reshape(problem.W, problem.K)


@pytest.fixture(scope="module")
def small():
    model = HeteroModel(seed=7, ny=2, nz_a=2, nz_b=4, n_layers=6, n_params=60)
    wmax = model.omega_max()
    om = (np.arange(24) + 0.5) * (1.05 * wmax / 24)
    kp = [(-2.0,), (0.3,), (2.9,)]
    return adjoint.HeteroKappaProblem(model, kp, om, 1e-6 * wmax * wmax, 300.0, 2 * np.pi * 15e12 / wmax)


def test_small_forward_matches_dense(small):
    theta = torch.as_tensor(small.model.theta0, device="cuda")
    t_gpu = small.transmission(theta)
    t_ref = dense_transmission(small, theta)
    assert float(t_ref.abs().max()) > 0.5
    err = float(((t_gpu - t_ref).abs() / t_ref.abs().clamp_min(1.0)).max())
    assert err < 1e-10, err


def test_kappa_grad_matches_dense_autograd(small):
    theta = torch.as_tensor(small.model.theta0, device="cuda").clone().requires_grad_(True)
    kap = adjoint.kappa(theta, small)
    (g_adj,) = torch.autograd.grad(kap, theta)
    theta_d = theta.detach().clone().requires_grad_(True)
    kap_d = small.kappa_of_t(dense_transmission(small, theta_d))
    (g_ref,) = torch.autograd.grad(kap_d, theta_d)
    assert abs(float(kap.detach() - kap_d.detach())) <= 1e-10 * abs(float(kap_d.detach()))
    scale = float(g_ref.abs().max())
    assert scale > 0
    err = float((g_adj - g_ref).abs().max()) / scale
    assert err < 1e-9, err


def test_vjp_random_weights_matches_dense_autograd(small):
    gen = torch.Generator(device="cpu").manual_seed(11)
    theta = torch.as_tensor(small.model.theta0, device="cuda") * (1 + 0.1 * torch.rand(
        small.model.theta0.size, generator=gen, dtype=torch.float64).cuda())
    w = torch.randn((small.W, small.K), generator=gen, dtype=torch.float64).cuda()
    th = theta.clone().requires_grad_(True)
    t = adjoint.TransmissionFunction.apply(th, small)
    (g_adj,) = torch.autograd.grad(t, th, grad_outputs=w)
    th_d = theta.clone().requires_grad_(True)
    (g_ref,) = torch.autograd.grad(dense_transmission(small, th_d), th_d, grad_outputs=w)
    err = float((g_adj - g_ref).abs().max()) / float(g_ref.abs().max())
    assert err < 1e-9, err


def test_zero_weights_give_zero_gradient(small):
    theta = torch.as_tensor(small.model.theta0, device="cuda")
    t, g = small.vjp(theta, torch.zeros((small.W, small.K), dtype=torch.float64, device="cuda"))
    assert float(g.abs().max()) == 0.0
    t_fwd = small.transmission(theta)
    assert float((t - t_fwd).abs().max()) < 1e-11


@pytest.fixture(scope="module")
def hetero():
    return adjoint.hetero_problem(n_k=4, n_omega=96)


def test_hetero_forward_matches_oracle(hetero):
    from oracle.negf_oracle import transmission_point

    m = hetero.model
    theta = torch.as_tensor(m.theta0, device="cuda")
    t = hetero.transmission(theta).cpu().numpy()
    on, cp = m.blocks(theta, hetero.kpoints)
    on, cp = on.cpu().numpy(), cp.cpu().numpy()
    la = m.lead_blocks("A", hetero.kpoints)
    lb = m.lead_blocks("B", hetero.kpoints)
    vl = hetero.vl.cpu().numpy()
    eta = float(hetero.eta[0])
    for wi, ki in [(10, 0), (40, 1), (70, 2), (90, 3)]:
        w = float(hetero.om[wi])
        ref = transmission_point(w, list(on[ki]), list(cp[ki]), (la["d00"][ki], la["d01"][ki], la["d10"][ki]),
                                 (lb["d00"][ki], lb["d01"][ki], lb["d10"][ki]), eta=eta, vl=vl[ki],
                                 vr=lb["d01"][ki])
        assert abs(t[wi, ki] - ref) <= 1e-10 * max(1.0, abs(ref)), (wi, ki, t[wi, ki], ref)


def test_hetero_grad_matches_central_differences(hetero):
    m = hetero.model
    assert m.n == 72 and m.n_a == 48 and m.L == 30 and m.theta0.size == 2000
    theta = torch.as_tensor(m.theta0, device="cuda")
    kap, g = hetero.kappa_and_grad(theta)
    rng = np.random.default_rng(5)
    sel = rng.choice(m.theta0.size, size=50, replace=False)
    h = 1e-6
    fd = []
    for p in sel:
        tp = theta.clone()
        tm = theta.clone()
        tp[p] += h
        tm[p] -= h
        fd.append(float(hetero.kappa_of_t(hetero.transmission(tp)) - hetero.kappa_of_t(hetero.transmission(tm)))
                  / (2 * h))
    fd = np.array(fd)
    ga = g.cpu().numpy()[sel]
    scale = np.abs(g.cpu().numpy()).max()
    err = np.abs(fd - ga) / scale
    assert scale > 0
    assert float(err.max()) < 1e-5, (float(err.max()), fd[:5], ga[:5])
    kap_fwd = hetero.kappa_of_t(hetero.transmission(theta))
    assert abs(float(kap - kap_fwd)) <= 1e-11 * abs(float(kap_fwd))
