"""Adjoint of the device solve: dkappa/dtheta, dkappa/dmasses and T
vector-Jacobian products.

Checked three ways: against torch autograd through a dense solve of the whole
device matrix (block order n = 24, the same lead surface GFs), against central
finite differences (h = 1e-6) of the forward kernels on 50 random spring
parameters and 20 random site masses of the heterojunction (lead 48 | 30
layers of order 72 | lead 72, 2000 spring parameters), and T of the
heterojunction against the oracle.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from negfpy_b200 import adjoint  # noqa: E402
from negfpy_b200.hetero import HeteroModel  # noqa: E402


def dense_transmission(problem, theta, masses=None):
    """T[W, K] by a dense solve of A = (w + i eta)^2 - D - Sigma over all layers (torch, differentiable)."""
    m = problem.model
    on, cp = m.blocks(theta, problem.kpoints, masses)
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
    pad = torch.zeros_like(A)
    pad[:, :n, :n] = sl
    pad[:, N - n:, N - n:] = sr
    A = A - pad
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


def _rel(a, b):
    return float((a - b).abs().max()) / float(b.abs().max())


def test_small_forward_matches_dense(small):
    theta = torch.as_tensor(small.model.theta0, device="cuda")
    t_gpu = small.transmission_theta(theta)
    t_ref = dense_transmission(small, theta)
    assert float(t_ref.abs().max()) > 0.5
    err = float(((t_gpu - t_ref).abs() / t_ref.abs().clamp_min(1.0)).max())
    assert err < 1e-10, err


def test_kappa_grads_match_dense_autograd(small):
    theta = torch.as_tensor(small.model.theta0, device="cuda").clone().requires_grad_(True)
    masses = torch.as_tensor(small.model.mass, device="cuda").clone().requires_grad_(True)
    kap = adjoint.kappa(theta, small, masses)
    g_th, g_m = torch.autograd.grad(kap, [theta, masses])
    th_d = theta.detach().clone().requires_grad_(True)
    m_d = masses.detach().clone().requires_grad_(True)
    kap_d = small.kappa_of_t(dense_transmission(small, th_d, m_d))
    r_th, r_m = torch.autograd.grad(kap_d, [th_d, m_d])
    assert abs(float(kap.detach() - kap_d.detach())) <= 1e-10 * abs(float(kap_d.detach()))
    assert float(r_th.abs().max()) > 0 and float(r_m.abs().max()) > 0
    assert _rel(g_th, r_th) < 1e-9
    assert _rel(g_m, r_m) < 1e-9
    # the one-launch path gives the same gradients
    k2, d_th, d_m = small.kappa_and_grad(theta.detach(), masses.detach())
    assert abs(float(k2 - kap_d.detach())) <= 1e-10 * abs(float(kap_d.detach()))
    assert _rel(d_th, r_th) < 1e-9 and _rel(d_m, r_m) < 1e-9


def test_vjp_random_weights_matches_dense_autograd(small):
    gen = torch.Generator(device="cpu").manual_seed(11)
    theta = torch.as_tensor(small.model.theta0, device="cuda") * (1 + 0.1 * torch.rand(
        small.model.theta0.size, generator=gen, dtype=torch.float64).cuda())
    w = torch.randn((small.W, small.K), generator=gen, dtype=torch.float64).cuda()
    th = theta.clone().requires_grad_(True)
    on, cp = small.blocks(th)
    t = adjoint.TransmissionFunction.apply(on, cp, small)
    (g_adj,) = torch.autograd.grad(t, th, grad_outputs=w)
    th_d = theta.clone().requires_grad_(True)
    (g_ref,) = torch.autograd.grad(dense_transmission(small, th_d), th_d, grad_outputs=w)
    assert _rel(g_adj, g_ref) < 1e-9


def test_zero_weights_give_zero_gradient(small):
    theta = torch.as_tensor(small.model.theta0, device="cuda")
    on, cp = small.blocks(theta)
    t, x_on, x_cp = small.vjp(on, cp, torch.zeros((small.W, small.K), dtype=torch.float64, device="cuda"))
    assert float(x_on.abs().max()) == 0.0 and float(x_cp.abs().max()) == 0.0
    t_fwd = small.transmission(on, cp)
    assert float((t - t_fwd).abs().max()) < 1e-11


@pytest.fixture(scope="module")
def hetero():
    return adjoint.hetero_problem(n_k=4, n_omega=96)


def test_hetero_forward_matches_oracle(hetero):
    from oracle.negf_oracle import transmission_point

    m = hetero.model
    theta = torch.as_tensor(m.theta0, device="cuda")
    t = hetero.transmission_theta(theta).cpu().numpy()
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


def test_hetero_grads_match_central_differences(hetero):
    m = hetero.model
    assert m.n == 72 and m.n_a == 48 and m.L == 30 and m.theta0.size == 2000
    theta = torch.as_tensor(m.theta0, device="cuda")
    masses = torch.as_tensor(m.mass, device="cuda")
    kap, g_th, g_m = hetero.kappa_and_grad(theta, masses)
    h = 1e-6
    kap_of = lambda th, ms: float(hetero.kappa_of_t(hetero.transmission_theta(th, ms)))  # noqa: E731
    rng = np.random.default_rng(5)
    # spring constants
    sel = rng.choice(m.theta0.size, size=50, replace=False)
    fd = []
    for p in sel:
        tp, tm = theta.clone(), theta.clone()
        tp[p] += h
        tm[p] -= h
        fd.append((kap_of(tp, masses) - kap_of(tm, masses)) / (2 * h))
    ga = g_th.cpu().numpy()
    err = np.abs(np.array(fd) - ga[sel]) / np.abs(ga).max()
    assert float(err.max()) < 1e-5, float(err.max())
    # site masses of the active device sites
    act = np.flatnonzero(m.active.ravel())
    msel = rng.choice(act, size=20, replace=False)
    fdm = []
    for q in msel:
        mp, mm = masses.clone().reshape(-1), masses.clone().reshape(-1)
        mp[q] += h
        mm[q] -= h
        fdm.append((kap_of(theta, mp.reshape(masses.shape)) - kap_of(theta, mm.reshape(masses.shape))) / (2 * h))
    gm = g_m.reshape(-1).cpu().numpy()
    errm = np.abs(np.array(fdm) - gm[msel]) / np.abs(gm).max()
    assert float(errm.max()) < 1e-5, float(errm.max())
    assert abs(float(kap) - kap_of(theta, masses)) <= 1e-11 * abs(float(kap))


def test_sharded_gradient_one_rank(hetero):
    """The omega-sharded gradient path (all-reduce over ranks) on one NCCL rank
    equals the unsharded one."""
    import os
    import socket

    import torch.distributed as dist

    from negfpy_b200.distributed import hetero_kappa_grad_sharded

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        m = hetero.model
        theta = torch.as_tensor(m.theta0, device="cuda")
        k, g_th, g_m = hetero_kappa_grad_sharded(m, hetero.kpoints, hetero.om.cpu().numpy(), hetero.eta0, theta,
                                                 None, hetero.temperature, hetero.omega_unit_rad_s)
        k0, g0, gm0 = hetero.kappa_and_grad(theta)
        assert abs(float(k) - float(k0)) <= 1e-13 * abs(float(k0))
        # the adjoint blocks are summed with FP64 atomics, in run-dependent order
        assert _rel(g_th, g0) < 1e-11 and _rel(g_m, gm0) < 1e-11
    finally:
        dist.destroy_process_group()
