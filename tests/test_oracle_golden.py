"""Pin the CPU oracle against negfpy's own outputs (tests/golden/*.npz)."""

import numpy as np
import pytest

from oracle import negf_oracle as O
from tests.conftest import GOLDEN, rel_err


def test_chain_transmission_matches_reference(golden):
    g = golden["chain"]
    L = int(g["n_layers"])
    lead = (np.array([[2.0]]), np.array([[-1.0]]), None)
    on = [np.array([[2.0]])] * L
    cp = [np.array([[-1.0]])] * (L - 1)
    idx = np.arange(0, 1000, 7)
    t = np.array([O.transmission_point(float(g["omegas"][i]), on, cp, lead, lead, eta=float(g["eta"])) for i in idx])
    assert np.max(rel_err(t, g["T"][idx])) < 1e-12


def test_chain_surface_gf_and_dos(golden):
    g = golden["chain"]
    for w, gref, dref in zip(g["g_omegas"], g["g"], g["dos"]):
        gs, _ = O.sancho_rubio(float(w), np.array([[2.0]]), np.array([[-1.0]]), None, 1e-8)
        assert abs(gs[0, 0] - gref) <= 1e-12 * max(abs(gref), 1.0)
        d = O.lead_surface_dos(float(w), np.array([[2.0]]), np.array([[-1.0]]), None, 1e-8)
        assert abs(d - dref) <= 1e-12 * max(abs(dref), 1.0)


def test_chain_kappa_matches_reference(golden):
    g = golden["chain"]
    k = O.thermal_conductance(g["omegas"], g["T"], g["temps"], float(g["omega_unit_rad_s"]))
    assert np.max(np.abs(k - g["kappa"]) / np.abs(g["kappa"])) < 1e-12


def _slab_args(g, i):
    wi, ki = g["pairs"][i]
    j = int(np.where(g["ksel"] == ki)[0][0])
    L = int(g["n_layers"])
    lead = (g["d00"][j], g["d01"][j], g["d10"][j])
    return float(g["omegas"][np.where(g["wsel"] == wi)[0][0]]), [g["onsite"][j]] * L, [g["coupling"][j]] * (L - 1), lead


def test_slab_transmission_matches_reference(golden):
    g = golden["slab"]
    for i in range(0, len(g["T"]), 5):
        w, on, cp, lead = _slab_args(g, i)
        t = O.transmission_point(w, on, cp, lead, lead, eta=float(g["eta"]))
        assert rel_err(t, g["T"][i]) < 1e-12


def test_slab_surface_gf_sr_and_qep(golden):
    g = golden["slab"]
    for (wi, ki), gref, gqep in zip(g["g_pts"], g["g"], g["g_qep"]):
        j = int(np.where(g["ksel"] == ki)[0][0])
        w = float(g["omegas"][np.where(g["wsel"] == wi)[0][0]])
        gs, it = O.sancho_rubio(w, g["d00"][j], g["d01"][j], g["d10"][j], float(g["eta"]))
        assert np.max(np.abs(gs - gref)) <= 1e-12 * np.max(np.abs(gref))
        gq = O.qep_surface_gf(w, g["d00"][j], g["d01"][j], g["d10"][j], float(g["eta"]))
        # two independent FP64 methods agree to the reference's own cross-check level
        assert np.max(np.abs(gq - gref)) <= 1e-7 * np.max(np.abs(gref))
        assert 1 <= it < 200


def test_reference_suite_cases(golden):
    c = golden["cases"]
    lead = (np.array([[2.0]]), np.array([[-1.0]]), None)
    on = [np.diag([2.0, 100.0]).astype(complex)] * 4
    cp = [np.diag([-1.0, 0.0]).astype(complex)] * 3
    t = O.transmission_point(1.0, on, cp, lead, lead, eta=1e-8, vl=np.array([[-1.0]]), vr=np.array([[-1.0]]),
                             idx_l=[0], idx_r=[6])
    assert rel_err(t, c["rect_T"]) < 1e-12
    assert 0.95 < t < 1.05
    for w, tr in zip(c["chain_plateau_omega"], c["chain_plateau_T"]):
        t = O.transmission_point(float(w), [np.array([[2.0]])] * 20, [np.array([[-1.0]])] * 19, lead, lead)
        assert rel_err(t, tr) < 1e-12


def test_oracle_error_cases():
    # maxiter exhausted
    with pytest.raises(O.OracleError):
        O.sancho_rubio(1.0, np.array([[2.0]]), np.array([[-1.0]]), None, 1e-8, maxiter=2)
    # exactly singular decimation block
    with pytest.raises(np.linalg.LinAlgError):
        O.sancho_rubio(1.0, np.eye(3), np.zeros((3, 3)), None, 0.0)


def test_bulk_n96_oracle_matches_reference():
    g = dict(np.load(__import__("tests.conftest", fromlist=["GOLDEN"]).GOLDEN / "bulk.npz"))
    L = int(g["n_layers"])
    for i in (0, 4):
        wi, ki = g["pairs"][i]
        j = int(np.where(g["ksel"] == ki)[0][0])
        w = float(g["omegas"][np.where(g["wsel"] == wi)[0][0]])
        d00, d01 = g["d00"][j], g["d01"][j]
        lead = (d00, d01, np.conj(d01).T)
        t = O.transmission_point(w, [d00] * L, [d01] * (L - 1), lead, lead, eta=float(g["eta"]))
        assert rel_err(t, g["T"][i]) < 1e-11


def test_oracle_failure_messages_follow_negfpy():
    """The oracle's decimation separates overflow from finite blocks
    ("numerically unstable") from NaN blocks ("non-finite values") as
    negfpy does (tests/golden/dos_workflow.npz holds negfpy's messages)."""
    import json

    from tests.golden.make_golden import SR_FAILURE_ORDERS, sr_failure_blocks

    ref = json.loads(str(np.load(GOLDEN / "dos_workflow.npz")["sr_failure_messages"]))
    for n in SR_FAILURE_ORDERS:
        for case, (d00, d01) in sr_failure_blocks(n).items():
            with pytest.raises(O.OracleError) as info:
                O.sancho_rubio(0.5, d00, d01, eta=1e-8)
            assert ref[f"{case}_{n}"].split(": ", 1)[1].startswith(str(info.value).rstrip("."))
