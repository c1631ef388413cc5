"""Heat current on the GPU against negfpy's values (tests/golden/thermal.npz)."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import negfpy_b200 as nb  # noqa: E402
from negfpy_b200 import thermal_current as TC  # noqa: E402


@pytest.fixture(scope="module")
def thermal():
    return np.load(Path(__file__).parent / "golden" / "thermal.npz")


def test_heat_current_from_spectrum(thermal):
    for (tl, tr), ref in zip(thermal["pairs"], thermal["j_spec"]):
        got = nb.heat_current_from_spectrum(thermal["om_rad"], thermal["t_chain"], tl, tr)
        if ref == 0.0:
            assert got == 0.0
        else:
            assert abs(got - ref) <= 1e-12 * abs(ref), (tl, tr, got, ref)
    rows = np.stack([thermal["t_chain"], 2.0 * thermal["t_chain"]])
    j = TC.heat_current_spectra(thermal["om_rad"], rows, 310.0, 290.0)
    assert abs(j[1] - 2.0 * j[0]) <= 1e-14 * abs(j[1])


def test_heat_current_1d_2d_3d(thermal):
    p = nb.ChainParams(1.0, 1.0)
    lead = nb.lead_blocks(p)
    j1 = nb.heat_current_1d(thermal["om1"], nb.device_perfect_chain(6, p), lead, lead, 1e-10, 0.5e-10, eta=1e-8)
    assert abs(j1 - float(thermal["j1"])) <= 1e-10 * abs(float(thermal["j1"]))
    from negfpy_b200.models import MaterialKspaceParams, material_kspace_device, material_kspace_lead

    # negfpy's square lattice (m = 1, spring_x = 1, spring_y = 0.5) as 1 x 1 force-constant terms
    fc00 = {(0, 0): np.array([[3.0]]), (1, 0): np.array([[-0.5]]), (-1, 0): np.array([[-0.5]])}
    fc01 = {(0, 0): np.array([[-1.0]])}
    prm = MaterialKspaceParams(masses=np.array([1.0]), fc00_terms=fc00, fc01_terms=fc01, dof_per_atom=1)
    kp = [tuple(k) for k in thermal["kp"]]
    lead = material_kspace_lead(prm)
    args = (thermal["om2"], material_kspace_device(5, prm), lead, lead, kp)
    j2 = nb.heat_current_per_length_2d(*args, 2.5, 2e-10, 1e-10, eta=1e-7)
    j3 = nb.heat_current_density_3d(*args, 4.0, 2e-10, 1e-10, eta=1e-7)
    assert abs(j2 - float(thermal["j2"])) <= 1e-10 * abs(float(thermal["j2"]))
    assert abs(j3 - float(thermal["j3"])) <= 1e-10 * abs(float(thermal["j3"]))


def test_fcs_cumulants_on_gpu(thermal):
    from negfpy_b200 import fcs

    t = thermal["t_chain"]
    for (tl, tr), ref in zip(thermal["pairs"], thermal["c_spec"]):
        c = fcs.heat_current_cumulants_from_spectrum(thermal["om_rad"], t, tl, tr)
        assert abs(c.c1_j_per_s - ref[0]) <= 1e-12 * max(abs(ref[0]), 1e-300)
        assert abs(c.c2_j2_per_s - ref[1]) <= 1e-12 * abs(ref[1])
    tw = thermal["t_wk"]
    c = fcs.heat_current_cumulants_from_k_moments(thermal["om2_rad"], tw.mean(1), (tw ** 2).mean(1), 300.0, 280.0)
    g = fcs.heat_current_cumulants_from_grid(thermal["om2_rad"], tw, 300.0, 280.0)
    for got in (c, g):
        assert abs(got.c1_j_per_s - thermal["c_mom"][0]) <= 1e-12 * abs(thermal["c_mom"][0])
        assert abs(got.c2_j2_per_s - thermal["c_mom"][1]) <= 1e-12 * abs(thermal["c_mom"][1])
    t1, t2 = fcs.k_moments(tw)
    np.testing.assert_allclose(t1.cpu().numpy(), tw.mean(1), rtol=1e-15, atol=0)
    np.testing.assert_allclose(t2.cpu().numpy(), (tw ** 2).mean(1), rtol=1e-15, atol=0)
