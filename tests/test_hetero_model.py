"""Host checks of the heterojunction model (no GPU): the device blocks of the
A and B regions reproduce the periodic leads, the blocks are Hermitian, the
leads are positive semidefinite and the contraction is the exact derivative
of a linear functional of the blocks."""

from __future__ import annotations

import numpy as np
import torch

from negfpy_b200.adjoint import kappa_weights
from negfpy_b200.hetero import HeteroModel

KP = [(-2.2,), (0.4,)]


def _blocks(m, theta=None):
    th = torch.as_tensor(m.theta0 if theta is None else theta, dtype=torch.float64)
    on, cp = m.blocks(th, KP)
    return on.numpy(), cp.numpy()


def test_sizes_of_the_differentiation_configuration():
    m = HeteroModel()
    assert (m.n_a, m.n, m.L, m.theta0.size) == (48, 72, 30, 2000)
    assert set(m.bond_la[m.param_bonds]) | set(m.bond_lb[m.param_bonds]) <= set(range(1, m.L - 1))


def test_regions_reproduce_the_leads():
    m = HeteroModel(seed=1, ny=2, nz_a=2, nz_b=3, n_layers=8, n_params=30)
    on, cp = _blocks(m)
    la, lb = m.lead_blocks("A", KP), m.lead_blocks("B", KP)
    ia = m.contact_left_indices()
    for l in range(1, m.split - 1):
        np.testing.assert_allclose(on[:, l][:, ia[:, None], ia], la["d00"], atol=1e-13)
        np.testing.assert_allclose(cp[:, l][:, ia[:, None], ia], la["d01"], atol=1e-13)
    np.testing.assert_allclose(on[:, 0][:, ia[:, None], ia], la["d00"], atol=1e-13)
    for l in range(m.split + 1, m.L):
        np.testing.assert_allclose(on[:, l], lb["d00"], atol=1e-13)
    np.testing.assert_allclose(cp[:, m.L - 2], lb["d01"], atol=1e-13)


def test_hermitian_and_psd():
    m = HeteroModel(seed=2, ny=2, nz_a=2, nz_b=3, n_layers=6, n_params=20)
    on, _ = _blocks(m)
    assert np.abs(on - np.conj(np.swapaxes(on, -1, -2))).max() < 1e-14
    for mat in ("A", "B"):
        lb = m.lead_blocks(mat, [(0.0,)])
        d = lb["d00"][0] + lb["d01"][0] + lb["d10"][0]  # kx = 0 bulk matrix
        assert np.linalg.eigvalsh(d).min() > -1e-12


def test_block_gradient_convention():
    """torch's gradient of F = 2 Re sum Tr[D X] with respect to complex D is
    2 conj(X^T): the form the adjoint's backward returns."""
    from negfpy_b200.adjoint import block_grads

    rng = np.random.default_rng(0)
    shape = (2, 3, 5, 5)
    X = torch.as_tensor(rng.normal(size=shape) + 1j * rng.normal(size=shape))
    Y = torch.as_tensor(rng.normal(size=shape) + 1j * rng.normal(size=shape))
    D = torch.zeros(shape, dtype=torch.complex128, requires_grad=True)
    C = torch.zeros(shape, dtype=torch.complex128, requires_grad=True)
    F = 2 * (torch.einsum("klab,klba->", D, X) + torch.einsum("klab,klba->", C, Y)).real
    gD, gC = torch.autograd.grad(F, [D, C])
    eD, eC = block_grads(X, Y)
    assert torch.allclose(gD, eD, rtol=0, atol=1e-14) and torch.allclose(gC, eC, rtol=0, atol=1e-14)


def test_blocks_are_differentiable_in_theta_and_masses():
    """Autograd of a linear functional of the blocks against central differences."""
    m = HeteroModel(seed=3, ny=2, nz_a=2, nz_b=3, n_layers=6, n_params=25)
    rng = np.random.default_rng(1)
    K, L, n = len(KP), m.L, m.n
    xo = torch.as_tensor(rng.normal(size=(K, L, n, n)) + 1j * rng.normal(size=(K, L, n, n)))
    xc = torch.as_tensor(rng.normal(size=(K, L - 1, n, n)) + 1j * rng.normal(size=(K, L - 1, n, n)))

    def F(th, ms):
        on, cp = m.blocks(th, KP, ms)
        return 2 * (torch.einsum("klab,klba->", on, xo) + torch.einsum("klab,klba->", cp, xc)).real

    th = torch.as_tensor(m.theta0, dtype=torch.float64).clone().requires_grad_(True)
    ms = torch.as_tensor(m.mass, dtype=torch.float64).clone().requires_grad_(True)
    g_th, g_m = torch.autograd.grad(F(th, ms), [th, ms])
    h = 1e-6
    for p in (0, 7, 24):
        tp, tm = th.detach().clone(), th.detach().clone()
        tp[p] += h
        tm[p] -= h
        fd = float(F(tp, ms.detach()) - F(tm, ms.detach())) / (2 * h)
        assert abs(fd - float(g_th[p])) <= 1e-6 * max(1.0, abs(fd))
    for q in (0, 5, 13, ms.numel() - 1):  # active and padding sites
        mp, mm = ms.detach().clone().reshape(-1), ms.detach().clone().reshape(-1)
        mp[q] += h
        mm[q] -= h
        fd = float(F(th.detach(), mp.reshape(ms.shape)) - F(th.detach(), mm.reshape(ms.shape))) / (2 * h)
        assert abs(fd - float(g_m.reshape(-1)[q])) <= 1e-6 * max(1.0, abs(fd))


def test_kappa_weights_trapezoid():
    om = torch.linspace(0.01, 3.0, 301, dtype=torch.float64)
    w = kappa_weights(om, 300.0, 1e13)
    # constant T = 1 integrates the Bose kernel; compare with a fine midpoint sum
    fine = torch.linspace(0.01, 3.0, 300001, dtype=torch.float64)
    wf = kappa_weights(fine, 300.0, 1e13)
    assert abs(float(w.sum() / wf.sum()) - 1) < 1e-4


def test_material_tables_default_to_the_model_and_build_the_leads():
    """The material spring tables reproduce the model's bonds and leads at
    their defaults; the torch lead builder equals the numpy one; equal
    parameters give bitwise-equal blocks."""
    m = HeteroModel(seed=7, ny=2, nz_a=2, nz_b=4, n_layers=6, n_params=60)
    th = torch.as_tensor(m.theta0, dtype=torch.float64)
    pa, pb = torch.as_tensor(m.phi0_a), torch.as_tensor(m.phi0_b)
    assert torch.equal(m.spring_values(th), m.spring_values(th, pa, pb))
    on0, cp0 = m.blocks(th, KP)
    on1, cp1 = m.blocks(th, KP, phi_a=pa, phi_b=pb)
    assert torch.equal(on0, on1) and torch.equal(cp0, cp1)
    for mat, phi in (("A", pa), ("B", pb)):
        ref = m.lead_blocks(mat, KP)
        got = m.lead_blocks_torch(mat, KP, phi)
        for key in ("d00", "d01", "d10"):
            assert np.abs(got[key].resolve_conj().numpy() - ref[key]).max() < 1e-14
        again = m.lead_blocks_torch(mat, KP, phi)
        assert torch.equal(got["d00"], again["d00"]) and torch.equal(got["d01"], again["d01"])


def test_material_table_reaches_lead_and_device():
    """A material-table entry moves the lead blocks and the device bonds of
    that material (a parameter shared by lead and device); theta overrides
    the bonds it owns."""
    m = HeteroModel(seed=7, ny=2, nz_a=2, nz_b=4, n_layers=6, n_params=60)
    th = torch.as_tensor(m.theta0, dtype=torch.float64)
    src, key = m.bond_src, m.bond_key
    free = [b for b in np.flatnonzero(src == 1) if not m.is_param[b]]
    q = int(key[free[0]])
    pa = torch.as_tensor(m.phi0_a).clone()
    pa[q] += 0.25
    kv0, kv1 = m.spring_values(th), m.spring_values(th, phi_a=pa)
    moved = np.flatnonzero((kv1 - kv0).abs().numpy() > 0)
    assert set(moved) == {b for b in np.flatnonzero((src == 1) & (key == q)) if not m.is_param[b]}
    la0, la1 = m.lead_blocks_torch("A", KP), m.lead_blocks_torch("A", KP, pa)
    assert float((la1["d00"] - la0["d00"]).abs().max()) > 0
