"""Heat current: the oracle against negfpy's values (tests/golden/thermal.npz),
and the host-side checks of the drop-in functions (no GPU)."""

from __future__ import annotations

import numpy as np
import pytest

from negfpy_b200 import thermal_current as TC
from oracle.negf_oracle import heat_current_from_spectrum as oracle_j


@pytest.fixture(scope="module")
def thermal(request):
    from pathlib import Path

    return np.load(Path(__file__).parent / "golden" / "thermal.npz")


def test_oracle_matches_reference(thermal):
    for (tl, tr), ref in zip(thermal["pairs"], thermal["j_spec"]):
        got = oracle_j(thermal["om_rad"], thermal["t_chain"], tl, tr)
        assert abs(got - ref) <= 1e-12 * max(abs(ref), 1e-300), (tl, tr, got, ref)


def test_transverse_length(thermal):
    assert abs(TC.transverse_length_from_vector([1.0, 2.0, 0.5], [0.0, 1.0, 0.0]) - float(thermal["tl"])) < 1e-15
    with pytest.raises(ValueError, match="non-zero"):
        TC.transverse_length_from_vector([1.0, 0.0], [0.0, 0.0])
    with pytest.raises(ValueError, match="orthogonal"):
        TC.transverse_length_from_vector([0.0, 2.0], [0.0, 1.0])
    with pytest.raises(ValueError, match="same size"):
        TC.transverse_length_from_vector([1.0, 0.0, 0.0], [0.0, 1.0])


def test_input_checks_match_negfpy():
    with pytest.raises(ValueError, match="at least two points"):
        TC.heat_current_from_spectrum([1.0], [1.0], 300.0, 290.0)
    with pytest.raises(ValueError, match="strictly increasing"):
        TC.heat_current_from_spectrum([1.0, 1.0, 2.0], [1.0, 1.0, 1.0], 300.0, 290.0)
    with pytest.raises(ValueError, match="same length"):
        TC.heat_current_from_spectrum([1.0, 2.0], [1.0], 300.0, 290.0)
    with pytest.raises(ValueError, match="positive in Kelvin"):
        TC.heat_current_from_spectrum([1.0, 2.0], [1.0, 1.0], 0.0, 290.0)
    with pytest.raises(ValueError, match="transverse_length must be positive"):
        TC.heat_current_per_length_2d([1.0, 2.0], None, None, None, [(0.0,)], 0.0, 300.0, 290.0)
    with pytest.raises(ValueError, match="transverse_area must be positive"):
        TC.heat_current_density_3d([1.0, 2.0], None, None, None, [(0.0,)], -1.0, 300.0, 290.0)


def test_fcs_oracle_matches_reference(thermal):
    from oracle.negf_oracle import fcs_cumulants

    t = thermal["t_chain"]
    for (tl, tr), ref in zip(thermal["pairs"], thermal["c_spec"]):
        c1, c2 = fcs_cumulants(thermal["om_rad"], t, t * t, tl, tr)
        assert abs(c1 - ref[0]) <= 1e-12 * max(abs(ref[0]), 1e-300)
        assert abs(c2 - ref[1]) <= 1e-12 * abs(ref[1])
    tw = thermal["t_wk"]
    c1, c2 = fcs_cumulants(thermal["om2_rad"], tw.mean(1), (tw ** 2).mean(1), 300.0, 280.0)
    assert abs(c1 - thermal["c_mom"][0]) <= 1e-12 * abs(thermal["c_mom"][0])
    assert abs(c2 - thermal["c_mom"][1]) <= 1e-12 * abs(thermal["c_mom"][1])


def test_fcs_host_checks_and_uncertainty(thermal):
    from negfpy_b200 import fcs

    with pytest.raises(ValueError, match="non-negative"):
        fcs.heat_current_cumulants_from_spectrum([1.0, 2.0], [1.0, -1.0], 300.0, 290.0)
    with pytest.raises(ValueError, match="match omega_rad_s shape"):
        fcs.heat_current_cumulants_from_k_moments([1.0, 2.0], [1.0], [1.0, 1.0], 300.0, 290.0)
    with pytest.raises(ValueError, match="Transmission moments must be non-negative"):
        fcs.heat_current_cumulants_from_k_moments([1.0, 2.0], [1.0, 1.0], [1.0, -1.0], 300.0, 290.0)
    with pytest.raises(ValueError, match="Temperature must be positive"):
        fcs.heat_current_cumulants_from_spectrum([1.0, 2.0], [1.0, 1.0], 300.0, -1.0)
    c = fcs.HeatCurrentCumulants(*thermal["c_mom"])
    u = fcs.heat_current_uncertainty(c, measurement_time_s=1e-6)
    np.testing.assert_allclose([u.std_current_j_per_s, u.variance_energy_j2, u.std_energy_j], thermal["unc"],
                               rtol=1e-14)
    with pytest.raises(ValueError, match="measurement_time_s must be positive"):
        fcs.heat_current_uncertainty(c, measurement_time_s=0.0)
