"""Host-side logic that needs no GPU: validation, embedding, workloads, no-fallback."""

import numpy as np
import pytest
import torch

import negfpy_b200 as nb
from negfpy_b200 import negf as N
from negfpy_b200 import workloads as W
from negfpy_b200.models import ChainParams, device_perfect_chain, lead_blocks
from negfpy_b200.surface_gf import check_method


def test_method_dispatch_matches_reference_names():
    for m in ("sancho_rubio", "Sancho-Rubio", " sr "):
        check_method(m)
    for m in ("generalized_eigen", "gep", "generalized_eigen_svd", "legacy"):
        with pytest.raises(NotImplementedError):
            check_method(m)
    with pytest.raises(ValueError, match="Unknown surface GF method"):
        check_method("bogus")


def test_point_system_default_contacts_embed_whole_layers():
    p = ChainParams(1.0, 1.0)
    s = N.point_system(1.0, device_perfect_chain(5, p), lead_blocks(p), lead_blocks(p), 1e-8)
    assert s["onsite"].shape == (5, 1, 1) and s["coupling"].shape == (4, 1, 1)
    assert s["vl"][0, 0] == -1.0 and s["vr"][0, 0] == -1.0


def test_point_system_rectangular_contacts():
    lead = nb.LeadBlocks(d00=np.array([[2.0]]), d01=np.array([[-1.0]]))
    on = [np.diag([2.0, 100.0]).astype(complex)] * 4
    cp = [np.diag([-1.0, 0.0]).astype(complex)] * 3
    s = N.point_system(1.0, nb.Device1D(on, cp), lead, lead, 1e-8, device_to_lead_left=np.array([[-1.0]]),
                       device_to_lead_right=np.array([[-1.0]]), contact_left_indices=[0], contact_right_indices=[6])
    assert s["vl"].shape == (2, 1) and s["vl"][0, 0] == -1.0 and s["vl"][1, 0] == 0.0
    assert s["vr"][0, 0] == -1.0 and s["vr"][1, 0] == 0.0


def test_point_system_errors_match_reference():
    p = ChainParams(1.0, 1.0)
    d, l = device_perfect_chain(4, p), lead_blocks(p)
    with pytest.raises(ValueError, match="eta_device must be non-negative"):
        N.point_system(1.0, d, l, l, 1e-8, eta_device=-1.0)
    with pytest.raises(ValueError, match="omega_scale must be positive"):
        N.point_system(1.0, d, l, l, 1e-8, omega_scale=0.0)
    with pytest.raises(ValueError, match="out of device range"):
        N.point_system(1.0, d, l, l, 1e-8, contact_left_indices=[9])
    with pytest.raises(ValueError, match="must be unique"):
        N.point_system(1.0, d, l, l, 1e-8, device_to_lead_left=np.ones((2, 1)), contact_left_indices=[0, 0])
    with pytest.raises(ValueError, match="Left contact index count"):
        N.point_system(1.0, d, l, l, 1e-8, contact_left_indices=[0, 1])
    with pytest.raises(ValueError, match="incompatible lead dimension"):
        N.point_system(1.0, d, l, l, 1e-8, device_to_lead_left=np.ones((1, 2)))
    with pytest.raises(ValueError, match="first principal layer"):
        N.point_system(1.0, d, l, l, 1e-8, contact_left_indices=[2])


def test_omega_scale_rescales_like_reference():
    p = ChainParams(1.0, 1.0)
    d, l = device_perfect_chain(3, p), lead_blocks(p)
    s = N.point_system(1.0, d, l, l, 1e-6, eta_device=2e-6, omega_scale=2.0)
    assert s["omega"] == 0.5 and s["eta"] == 5e-7 and s["eta_dev"] == 1e-6
    assert s["onsite"][0, 0, 0] == 0.5
    # the default couplings are divided by s^2 once more, as negfpy does
    assert s["vl"][0, 0] == -1.0 / 16.0


def test_adaptive_argument_checks():
    p = ChainParams(1.0, 1.0)
    d, l = device_perfect_chain(4, p), lead_blocks(p)
    with pytest.raises(ValueError, match="kpoints must contain"):
        nb.transmission_kavg_adaptive(1.0, d, l, l, kpoints=[])
    with pytest.raises(ValueError, match="eta_values must contain"):
        nb.transmission_kavg_adaptive(1.0, d, l, l, kpoints=[()], eta_values=())
    with pytest.raises(ValueError, match="min_success_fraction"):
        nb.transmission_kavg_adaptive_global_eta(1.0, d, l, l, kpoints=[()], min_success_fraction=2.0)


def test_spring_network_is_psd_hermitian_and_obeys_asr():
    params = W.spring_network(7, ny=2, nz=3, periodic_y=True, periodic_z=False)
    st = nb.models.material_kspace_stack(params, [(0.3,), (-1.1,)])
    for k in range(2):
        d00, d01, d10 = st["d00"][k], st["d01"][k], st["d10"][k]
        assert np.allclose(d00, d00.conj().T, atol=1e-14)
        assert np.allclose(d10, d01.conj().T, atol=1e-14)
        for kx in (0.0, 0.7, np.pi):
            dk = d00 + d01 * np.exp(1j * kx) + d10 * np.exp(-1j * kx)
            assert np.linalg.eigvalsh(dk).min() > -1e-12
    # acoustic sum rule: at k = 0 the summed force constants annihilate uniform translations
    phi = sum(params.fc00_terms.values()) + sum(params.fc01_terms.values()) + sum(
        b.T for b in params.fc01_terms.values())
    u = np.tile(np.eye(3), (params.n_atoms, 1))
    assert np.max(np.abs(phi @ u)) < 1e-12


def test_workloads_shapes_and_grids():
    wl = W.slab_workload(n_omega=16, n_k=4)
    assert wl.n == 48 and wl.onsite.shape == (4, 1, 48, 48) and len(wl.kpoints) == 4
    assert np.all(np.diff(wl.omegas) > 0) and np.isclose(wl.omegas[-1], 1.05 * wl.omega_max)
    assert np.isclose(wl.eta, 1e-6 * wl.omega_max ** 2)
    ks = W.kline(64)
    assert np.isclose(ks[0], -np.pi + np.pi / 64) and np.allclose(ks, -ks[::-1])
    ch = W.chain_workload()
    assert ch.n == 1 and len(ch.omegas) == 1000 and 0 < ch.omegas[0] < ch.omegas[-1] < 2.0


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU behaviour")
def test_no_cpu_fallback_without_gpu():
    p = ChainParams(1.0, 1.0)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        nb.transmission(1.0, device_perfect_chain(4, p), lead_blocks(p), lead_blocks(p))
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        nb.surface_gf(1.0, np.array([[2.0]]), np.array([[-1.0]]))
