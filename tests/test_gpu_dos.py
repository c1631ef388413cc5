"""k-averaged, adaptive and spectrum forms of the lead surface DOS against
negfpy's own (core/dos.py:64-252, tests/golden/dos.npz), on a 2D-k material
lead (n = 12) and on the two different leads of its interface contacts.

Tolerance: 1e-9 max(|DOS_ref|, 1), as for the single-point DOS (a trace of
Im g, less well conditioned than T).  For the adaptive forms one k point has
NaN blocks, so it fails at every eta; the ladder statistics must match
negfpy's exactly.  (A ladder that starts at eta = 0 is not a usable check:
with a real z the decimation's outcome at some k points depends on
rounding, and negfpy itself "converges" there to a negative DOS.)
"""

from __future__ import annotations

import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import negfpy_b200 as nb  # noqa: E402
from negfpy_b200.models import interface_contacts, material_kspace_lead  # noqa: E402
from negfpy_b200.types import LeadKSpace  # noqa: E402
from tests.conftest import GOLDEN, rel_err  # noqa: E402
from tests.golden.make_golden import DOS_KPOINTS, poisoned_blocks  # noqa: E402
from tests.test_gpu_workflow import _close  # noqa: E402
from tests.test_interface_host import params_of  # noqa: E402

TOL_DOS = 1e-9


@pytest.fixture(scope="module")
def setup():
    fix = np.load(GOLDEN / "dos.npz")
    prm = params_of(np.load(GOLDEN / "interface.npz"), "bulk")
    return fix, prm, material_kspace_lead(prm)


def _poisoned(lead):
    return LeadKSpace(blocks_builder=lambda k: poisoned_blocks(lead, k))


def test_kavg_matches_negfpy(setup):
    fix, prm, lead = setup
    eta = float(fix["eta"])
    got = [nb.lead_surface_dos_kavg(float(w), lead, DOS_KPOINTS, eta) for w in fix["omegas"]]
    assert rel_err(got, fix["kavg"]).max() <= TOL_DOS
    got = [nb.lead_surface_dos_kavg(float(w), lead, DOS_KPOINTS, eta, normalize_per_mode=True) for w in fix["omegas"]]
    assert rel_err(got, fix["kavg_norm"]).max() <= TOL_DOS


def test_adaptive_ladder_matches_negfpy(setup):
    fix, prm, lead = setup
    ladder = tuple(float(x) for x in fix["ladder"])
    ref_info = json.loads(str(fix["adaptive_info"]))
    for i, w in enumerate(fix["omegas"]):
        v, info = nb.lead_surface_dos_kavg_adaptive(float(w), _poisoned(lead), DOS_KPOINTS, ladder, 0.5)
        assert rel_err(v, fix["adaptive"][i]) <= TOL_DOS, i
        _close(json.loads(json.dumps(info)), ref_info[i], TOL_DOS)


def test_spectra_match_negfpy(setup):
    fix, prm, lead = setup
    om, eta = fix["omegas"], float(fix["eta"])
    ladder = tuple(float(x) for x in fix["ladder"])
    assert rel_err(nb.lead_surface_dos_spectrum(om, lead, kpoints=DOS_KPOINTS, eta=eta), fix["spectrum_k"]).max() <= TOL_DOS
    assert rel_err(nb.lead_surface_dos_spectrum(om, _poisoned(lead), kpoints=DOS_KPOINTS, eta_values=ladder,
                                                min_success_fraction=0.5), fix["spectrum_ladder"]).max() <= TOL_DOS
    assert rel_err(nb.lead_surface_dos_spectrum(om, lead, eta=eta), fix["spectrum_gamma"]).max() <= TOL_DOS
    ll, lr, _, _ = interface_contacts(prm)
    two = nb.leads_surface_dos_spectrum(om, ll, lr, kpoints=DOS_KPOINTS, eta=eta, normalize_per_mode=True)
    assert rel_err(two["left"], fix["leads_left"]).max() <= TOL_DOS
    assert rel_err(two["right"], fix["leads_right"]).max() <= TOL_DOS
