"""GPU parity: CUDA path vs negfpy's own outputs (golden) and vs the CPU oracle.

Tolerance for the FP64 path: |T_gpu - T_ref| <= 1e-10 * max(|T_ref|, 1);
surface DOS: 1e-9 * max(|DOS_ref|, 1).
"""

import numpy as np
import pytest
import torch

import negfpy_b200 as nb
from negfpy_b200 import _lib, engine
from negfpy_b200 import workloads as W
from negfpy_b200.models import ChainParams, device_perfect_chain, lead_blocks
from oracle import negf_oracle as O
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu
TOL_T = 1e-10
TOL_DOS = 1e-9


def _slab_system(g, j, L=None):
    L = int(g["n_layers"]) if L is None else L
    lead = nb.LeadBlocks(d00=g["d00"][j], d01=g["d01"][j], d10=g["d10"][j])
    dev = nb.Device1D([g["onsite"][j]] * L, [g["coupling"][j]] * (L - 1))
    return lead, dev


def test_chain_transmission_grid_matches_reference(golden):
    g = golden["chain"]
    p = ChainParams(1.0, 1.0)
    r = nb.transmission_grid(g["omegas"], None, device_perfect_chain(int(g["n_layers"]), p), lead_blocks(p),
                             lead_blocks(p), eta=float(g["eta"]))
    assert np.all(r["status"] == 0)
    err = rel_err(r["T"][:, 0], g["T"])
    assert err.max() <= TOL_T, (err.max(), int(err.argmax()))


def test_chain_surface_gf_and_dos(golden):
    g = golden["chain"]
    lead = lead_blocks(ChainParams(1.0, 1.0))
    for w, gref, dref in zip(g["g_omegas"], g["g"], g["dos"]):
        gs = nb.surface_gf(float(w), lead.d00, lead.d01, eta=1e-8)
        assert abs(gs[0, 0] - gref) <= 1e-12 * max(abs(gref), 1.0)
        d = nb.lead_surface_dos(float(w), lead, eta=1e-8)
        assert abs(d - dref) <= 1e-12 * max(abs(dref), 1.0)


def test_chain_kappa_matches_reference(golden):
    g = golden["chain"]
    k = nb.thermal_conductance_from_spectrum(g["omegas"], g["T"], g["temps"], float(g["omega_unit_rad_s"]))
    assert np.max(np.abs(k - g["kappa"]) / np.abs(g["kappa"])) < 1e-12


def test_slab_surface_gf_matches_reference(golden):
    g = golden["slab"]
    for (wi, ki), gref in zip(g["g_pts"], g["g"]):
        j = int(np.where(g["ksel"] == ki)[0][0])
        w = float(g["omegas"][np.where(g["wsel"] == wi)[0][0]])
        gs = nb.surface_gf(w, g["d00"][j], g["d01"][j], g["d10"][j], eta=float(g["eta"]))
        assert np.max(np.abs(gs - gref)) <= 1e-10 * np.max(np.abs(gref))


def test_slab_transmission_and_dos_match_reference(golden):
    g = golden["slab"]
    ts, ds = [], []
    for i, (wi, ki) in enumerate(g["pairs"]):
        j = int(np.where(g["ksel"] == ki)[0][0])
        w = float(g["omegas"][np.where(g["wsel"] == wi)[0][0]])
        lead, dev = _slab_system(g, j)
        ts.append(nb.transmission(w, dev, lead, lead, eta=float(g["eta"])))
        ds.append(nb.lead_surface_dos(w, lead, eta=float(g["eta"])))
    assert rel_err(ts, g["T"]).max() <= TOL_T
    # The DOS is a trace of Im g; it is less well conditioned than T, and two
    # FP64 implementations (LAPACK LU vs Gauss-Jordan) differ by up to a few
    # 1e-10 relative near resonances.  Tolerance: 1e-9 * max(|DOS_ref|, 1).
    assert rel_err(ds, g["dos"]).max() <= TOL_DOS


def test_reference_suite_cases_on_gpu(golden):
    c = golden["cases"]
    p = ChainParams(1.0, 1.0)
    l = lead_blocks(p)
    t = [nb.transmission(float(w), device_perfect_chain(20, p), l, l, eta=1e-8) for w in c["chain_plateau_omega"]]
    assert rel_err(t, c["chain_plateau_T"]).max() <= TOL_T
    assert np.mean(t) > 0.96 and np.max(np.abs(np.array(t) - 1.0)) < 0.08
    t = [nb.transmission(float(w), device_perfect_chain(16, p), l, l, eta=1e-8) for w in c["chain_outband_omega"]]
    assert np.max(np.abs(np.array(t) - c["chain_outband_T"])) <= 1e-12 and np.max(np.abs(t)) < 1e-4
    lead1 = nb.LeadBlocks(d00=np.array([[2.0]], dtype=complex), d01=np.array([[-1.0]], dtype=complex))
    on = [np.diag([2.0, 100.0]).astype(complex)] * 4
    cp = [np.diag([-1.0, 0.0]).astype(complex)] * 3
    t = nb.transmission(1.0, nb.Device1D(on, cp), lead1, lead1, eta=1e-8, device_to_lead_left=np.array([[-1.0]]),
                        device_to_lead_right=np.array([[-1.0]]), contact_left_indices=[0], contact_right_indices=[6])
    assert rel_err(t, c["rect_T"]) <= TOL_T
    md = np.eye(6)
    lead6 = nb.LeadBlocks(d00=2.0 * md, d01=-md)
    t = nb.transmission(1.0, nb.Device1D([2.0 * md] * 30, [-md] * 29), lead6, lead6, eta=1e-8)
    assert rel_err(t, c["multidof_T"]) <= TOL_T and 0.95 * 6 < t < 1.05 * 6
    tav, info = nb.transmission_kavg_adaptive(1.0, device_perfect_chain(14, p), l, l, kpoints=[(), (), ()],
                                              eta_values=(1e-8, 1e-7), min_success_fraction=1.0)
    assert rel_err(tav, c["chain_adaptive_T"]) <= TOL_T
    assert info["n_success"] == 3 and info["n_failed"] == 0


def test_omega_scale_and_device_eta(golden):
    c, g = golden["cases"], golden["slab"]
    j = int(np.where(g["ksel"] == 13)[0][0])
    lead, dev = _slab_system(g, j, L=6)
    w = float(g["omegas"][np.where(g["wsel"] == 900)[0][0]])
    t = nb.transmission(w, dev, lead, lead, eta=float(g["eta"]), eta_device=3.0 * float(g["eta"]), omega_scale=1.7)
    assert rel_err(t, c["slab_scaled_T"]) <= TOL_T


def test_kspace_square_lattice_kavg(golden):
    from negfpy_b200.models import MaterialKspaceParams, material_kspace_device, material_kspace_lead

    c = golden["cases"]
    # square lattice m=1, kx=1, ky=0.5 as 1x1 force-constant terms
    fc00 = {(0, 0): np.array([[3.0]]), (1, 0): np.array([[-0.5]]), (-1, 0): np.array([[-0.5]])}
    fc01 = {(0, 0): np.array([[-1.0]])}
    prm = MaterialKspaceParams(masses=np.array([1.0]), fc00_terms=fc00, fc01_terms=fc01, dof_per_atom=1)
    kp = [tuple(k) for k in c["square_kpoints"]]
    lead, dev = material_kspace_lead(prm), material_kspace_device(25, prm)
    t = [nb.transmission(0.9, dev, lead, lead, kpar=k) for k in kp]
    assert rel_err(t, c["square_T"]).max() <= TOL_T
    assert rel_err(nb.transmission_kavg(0.9, dev, lead, lead, kpoints=kp), c["square_kavg"]) <= TOL_T


def test_status_codes_for_failures():
    dev = _lib.require_cuda()
    # exactly singular decimation block: d00 = z, d01 = 0 at eta = 0
    n = 6
    d00 = torch.eye(n, dtype=torch.complex128, device=dev)
    d01 = torch.zeros(n, n, dtype=torch.complex128, device=dev)
    om = torch.tensor([1.0], dtype=torch.float64, device=dev)
    et = torch.tensor([0.0], dtype=torch.float64, device=dev)
    r = engine.sgf_sr(d00, d01, None, om, et)
    assert int(r["status"][0]) == _lib.SINGULAR
    # maxiter exhausted
    l = lead_blocks(ChainParams(1.0, 1.0))
    with pytest.raises(RuntimeError, match="did not converge"):
        nb.surface_gf_sancho_rubio(1.0, l.d00, l.d01, eta=1e-8, maxiter=2)
    # non-finite input
    bad = np.full((4, 4), np.nan, dtype=complex)
    with pytest.raises(RuntimeError, match="non-finite"):
        nb.surface_gf(1.0, bad, bad)
    with pytest.raises(np.linalg.LinAlgError):
        nb.surface_gf(1.0, np.eye(3), np.zeros((3, 3)), eta=0.0)


def test_slab_full_grid_properties_and_oracle_sample():
    """c2 at full size (2048 x 64 points): size-independent checks plus an oracle sample.

    Checks: every point converges; 0 <= T (Gamma_L, Gamma_R are positive
    semidefinite) and T below the channel count n; results do not depend on
    the batch layout (a permuted batch gives bitwise the same T); a random
    sample agrees with the oracle to the FP64 tolerance.  (T(k) = T(-k) is
    NOT a property of negfpy's formula: it builds the left lead's surface GF
    with the same decimation direction as the right one.)
    """
    wl = W.slab_workload()
    s = engine.StackedSystem.from_arrays(wl.lead_l, wl.lead_l, wl.onsite, wl.coupling, wl.n_layers)
    dev = _lib.require_cuda()
    K, Wn = len(wl.kpoints), len(wl.omegas)
    wi = torch.arange(Wn, device=dev).repeat_interleave(K)
    ki = torch.arange(K, device=dev, dtype=torch.int32).repeat(Wn)
    om = torch.tensor(wl.omegas, device=dev)[wi]
    eta = torch.full_like(om, wl.eta)
    r = s.transmission(om, ki, eta)
    T = r["T"].reshape(Wn, K).cpu().numpy()
    st = r["status"].cpu().numpy()
    assert np.all(st == 0)
    assert T.min() > -1e-8 and T.max() < wl.n + 1e-6
    perm = torch.randperm(Wn * K, device=dev, generator=torch.Generator(device=dev).manual_seed(3))
    rp = s.transmission(om[perm], ki[perm], eta[perm])
    Tp = torch.empty_like(rp["T"])
    Tp[perm] = rp["T"]
    assert torch.equal(Tp.reshape(Wn, K).cpu(), torch.as_tensor(T))
    rng = np.random.default_rng(11)
    pairs = [(int(a), int(b)) for a, b in zip(rng.integers(0, Wn, 6), rng.integers(0, K, 6))]
    ref = O.transmission_points(wl, pairs)
    got = np.array([T[a, b] for a, b in pairs])
    assert rel_err(got, ref).max() <= TOL_T


@pytest.mark.parametrize("n", [3, 16, 29, 40, 47, 48])
@pytest.mark.parametrize("scale", [1e-200, 1e-3, 1.0, 1e5, 1e200])
def test_inversion_against_numpy(n, scale):
    """With d01 = 0 the decimation ends after one sweep with g = (z - d00)^-1,
    a direct check of the in-kernel Gauss-Jordan inverse (pivot search and the
    division-free pivot reciprocal) against LAPACK, over 400 orders of
    magnitude of entry size.  Tolerance: 1e-12 * cond(z - d00)."""
    rng = np.random.default_rng(n)
    d00 = (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))) * scale
    z = (0.7 + 1j * 0.01) ** 2
    m = z * np.eye(n) - d00
    ref = np.linalg.inv(m)
    g = nb.surface_gf(0.7, d00, np.zeros((n, n)), eta=0.01)
    err = np.max(np.abs(g - ref)) / np.max(np.abs(ref))
    assert err <= 1e-12 * np.linalg.cond(m), err


# ------------------------------------------------ block orders above 48 ----
def test_bulk_n96_matches_reference(golden_bulk):
    """n = 96, L = 40 (the bulk configuration): global-memory kernels vs negfpy."""
    g = golden_bulk
    L = int(g["n_layers"])
    ts = []
    for wi, ki in g["pairs"]:
        j = int(np.where(g["ksel"] == ki)[0][0])
        w = float(g["omegas"][np.where(g["wsel"] == wi)[0][0]])
        d00, d01 = g["d00"][j], g["d01"][j]
        lead = nb.LeadBlocks(d00=d00, d01=d01, d10=np.conj(d01).T)
        dev = nb.Device1D([d00] * L, [d01] * (L - 1))
        ts.append(nb.transmission(w, dev, lead, lead, eta=float(g["eta"])))
    assert rel_err(ts, g["T"]).max() <= TOL_T
    w = float(g["omegas"][np.where(g["wsel"] == 1700)[0][0]])
    gs = nb.surface_gf(w, g["d00"][0], g["d01"][0], np.conj(g["d01"][0]).T, eta=float(g["eta"]))
    assert np.max(np.abs(gs - g["g"])) <= 1e-10 * np.max(np.abs(g["g"]))


@pytest.mark.parametrize("n", [49, 64, 96, 150, 192, 256])
def test_inversion_large_orders_against_numpy(n):
    rng = np.random.default_rng(n)
    d00 = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    z = (0.7 + 1j * 0.01) ** 2
    m = z * np.eye(n) - d00
    ref = np.linalg.inv(m)
    g = nb.surface_gf(0.7, d00, np.zeros((n, n)), eta=0.01)
    err = np.max(np.abs(g - ref)) / np.max(np.abs(ref))
    assert err <= 1e-12 * np.linalg.cond(m), err


def test_padded_order_48_transmission_vs_oracle():
    """n = 42 (14 atoms x 3 DOF) runs on the n = 48 kernels with 6 padding
    rows and columns: T against the oracle at four (omega, k) points."""
    from negfpy_b200.models import material_kspace_device, material_kspace_lead

    p = W.spring_network(6, ny=2, nz=7, periodic_y=True, periodic_z=False)
    assert p.ndof == 42
    wmax = W.estimate_omega_max(p, nk=6)
    eta = 1e-5 * wmax * wmax
    kp = [(0.9,), (-2.4,)]
    lead, dev = material_kspace_lead(p), material_kspace_device(7, p)
    om = np.array([0.31, 0.67]) * wmax
    r = nb.transmission_grid(om, kp, dev, lead, lead, eta=eta)
    assert np.all(r["status"] == 0)
    for wi in range(2):
        for ki in range(2):
            d = dev.device(kp[ki])
            lb = lead.blocks(kp[ki])
            ref = O.transmission_point(float(om[wi]), list(d.onsite_blocks), list(d.coupling_blocks), lb, lb, eta=eta)
            assert abs(r["T"][wi, ki] - ref) <= TOL_T * max(1.0, abs(ref)), (wi, ki, r["T"][wi, ki], ref)


def test_largest_block_order_transmission_vs_oracle():
    """n = 255 (85 atoms x 3 DOF, padded to the largest supported order 256):
    T through the global-workspace kernels against the oracle at three
    (omega, k) points, and order 257 is rejected."""
    from negfpy_b200.models import material_kspace_device, material_kspace_lead

    p = W.spring_network(4, ny=5, nz=17, periodic_y=True, periodic_z=False)
    assert p.ndof == 255
    wmax = W.estimate_omega_max(p, nk=4)
    eta = 1e-5 * wmax * wmax
    kp = [(0.4,), (-2.1,)]
    lead, dev = material_kspace_lead(p), material_kspace_device(3, p)
    om = np.array([0.23, 0.61]) * wmax
    r = nb.transmission_grid(om, kp, dev, lead, lead, eta=eta)
    assert np.all(r["status"] == 0)
    for wi, ki in ((0, 0), (1, 0), (1, 1)):
        d = dev.device(kp[ki])
        lb = lead.blocks(kp[ki])
        ref = O.transmission_point(float(om[wi]), list(d.onsite_blocks), list(d.coupling_blocks), lb, lb, eta=eta)
        assert abs(r["T"][wi, ki] - ref) <= TOL_T * max(1.0, abs(ref)), (wi, ki, r["T"][wi, ki], ref)
    big = np.eye(257, dtype=complex)
    with pytest.raises(RuntimeError, match="block order 257 is not supported"):
        nb.surface_gf(0.5, big, np.zeros_like(big), eta=0.01)


def test_mixed_orders_heterojunction_vs_oracle():
    """Left lead n = 48, right lead n = 72, device blocks of order 72 with the
    left contact on the first 48 DOFs (rectangular couplings, explicit contact
    indices), against the CPU oracle."""
    left = W.spring_network(21, ny=2, nz=8, periodic_y=True)
    right = W.spring_network(22, ny=3, nz=8, periodic_y=True, spring_range=(0.8, 1.6), mass_range=(0.9, 1.4))
    from negfpy_b200.models import material_kspace_stack

    kp = [(0.4,)]
    sl = material_kspace_stack(left, kp)
    sr = material_kspace_stack(right, kp, n_layers=5)
    L = 5
    on = [sr["onsite"][0, i] for i in range(L)]
    cp = [sr["coupling"][0, i] for i in range(L - 1)]
    ll = (sl["d00"][0], sl["d01"][0], sl["d10"][0])
    lr = (sr["d00"][0], sr["d01"][0], sr["d10"][0])
    vl = np.zeros((48, 48), dtype=complex)
    vl[:, :] = 0.8 * sl["d10"][0]
    idx_l = list(range(48))
    idx_r = list(range(72 * (L - 1), 72 * L))
    for w in (0.9, 1.7, 2.6):
        ref = O.transmission_point(w, on, cp, ll, lr, eta=1e-4, vl=vl, vr=lr[1], idx_l=idx_l, idx_r=idx_r)
        t = nb.transmission(w, nb.Device1D(on, cp), nb.LeadBlocks(*ll), nb.LeadBlocks(*lr), eta=1e-4,
                            device_to_lead_left=vl, device_to_lead_right=lr[1], contact_left_indices=idx_l,
                            contact_right_indices=idx_r)
        assert rel_err(t, ref) <= TOL_T, (w, t, ref)
