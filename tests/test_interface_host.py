"""The IFC transport set-up of negfpy's workflow (``_build_interface_contacts``,
``workflows/ifc_bulk.py:690-742``) on the host: blocks and couplings against
negfpy's own (``tests/golden/interface.npz``), the dispatch of the batched
path, and the oracle's T through these contacts against negfpy's."""

from __future__ import annotations

import numpy as np
import pytest

from negfpy_b200 import workflow
from negfpy_b200.models import (MaterialKspaceParams, interface_contacts, interface_terms, material_kspace_device,
                                material_kspace_lead)
from negfpy_b200.spectrum import _material_fast_path

NAMES = ("slab", "bulk")


@pytest.fixture(scope="module")
def fix():
    from tests.conftest import GOLDEN

    return np.load(GOLDEN / "interface.npz")


def params_of(fix, name: str) -> MaterialKspaceParams:
    def terms(prefix):
        if prefix + "_keys" not in fix.files:
            return None
        return {tuple(int(x) for x in k): b for k, b in zip(fix[prefix + "_keys"], fix[prefix + "_blocks"])}

    return MaterialKspaceParams(masses=fix[f"{name}_masses"], fc00_terms=terms(f"{name}_fc00"),
                                fc01_terms=terms(f"{name}_fc01"), fc10_terms=terms(f"{name}_fc10"),
                                dof_per_atom=3, onsite_pinning=float(fix[f"{name}_pinning"]))


def kpoints_of(name: str):
    from tests.golden.make_golden import INTERFACE_KPOINTS

    return INTERFACE_KPOINTS[name]


@pytest.mark.parametrize("name", NAMES)
def test_blocks_match_negfpy(fix, name):
    ll, lr, vdl_l, vdl_r = interface_contacts(params_of(fix, name))
    for j, k in enumerate(kpoints_of(name)):
        for side, lead in (("l", ll), ("r", lr)):
            b = lead.blocks(k)
            for i, key in enumerate(("d00", "d01", "d10")):
                ref = fix[f"{name}_{side}_{key}"][j]
                assert np.abs(b[i] - ref).max() <= 1e-15 * np.abs(ref).max(), (name, side, key, k)
        for got, key in ((vdl_l(k), "vl"), (vdl_r(k), "vr")):
            ref = fix[f"{name}_{key}"][j]
            assert np.abs(got - ref).max() <= 1e-15 * np.abs(ref).max(), (name, key, k)


def test_workflow_alias_and_terms(fix):
    assert workflow._build_interface_contacts is interface_contacts
    prm = params_of(fix, "slab")
    left, right = interface_terms(prm)
    assert set(right) == {(-dy, -dz) for dy, dz in left}
    for (dy, dz), v in left.items():
        assert np.array_equal(right[(-dy, -dz)], v.T)
    # without fc10 terms the left terms are FC01^H at the negated shift
    for (dy, dz), v in prm.fc01_terms.items():
        assert np.array_equal(left[(-dy, -dz)], np.asarray(v, dtype=complex).conj().T)


def test_fast_path_dispatch(fix):
    prm = params_of(fix, "slab")
    dev = material_kspace_device(4, prm)
    ll, lr, vl, vr = interface_contacts(prm)
    kind = _material_fast_path(dev, ll, lr, vl, vr, None, None, None)
    assert kind is not None and kind[0] == "interface" and kind[1] is prm
    # pieces of two different set-ups, a missing coupling, explicit contacts or an omega scale: host path
    ll2, lr2, vl2, vr2 = interface_contacts(prm)
    assert _material_fast_path(dev, ll, lr2, vl, vr, None, None, None) is None
    assert _material_fast_path(dev, ll, lr, vl, None, None, None, None) is None
    assert _material_fast_path(dev, ll, lr, vl, vr, [0, 1], None, None) is None
    assert _material_fast_path(dev, ll, lr, vl, vr, None, None, 2.0) is None
    # a device of other parameters
    other = MaterialKspaceParams(masses=prm.masses * 1.5, fc00_terms=prm.fc00_terms, fc01_terms=prm.fc01_terms)
    assert _material_fast_path(material_kspace_device(4, other), ll, lr, vl, vr, None, None, None) is None
    # material leads with default couplings
    lead = material_kspace_lead(prm)
    assert _material_fast_path(dev, lead, lead, None, None, None, None, None)[0] == "material"
    # complex force constants stay on the host builder
    cplx = MaterialKspaceParams(masses=prm.masses, fc00_terms=prm.fc00_terms,
                                fc01_terms={k: v * (1 + 1e-3j) for k, v in prm.fc01_terms.items()})
    lc = material_kspace_lead(cplx)
    assert _material_fast_path(material_kspace_device(4, cplx), lc, lc, None, None, None, None, None) is None


@pytest.mark.parametrize("name", NAMES)
def test_oracle_transmission_matches_negfpy(fix, name):
    from oracle.negf_oracle import transmission_point

    from tests.golden.make_golden import INTERFACE_LAYERS

    prm = params_of(fix, name)
    L = INTERFACE_LAYERS[name]
    dev = material_kspace_device(L, prm)
    eta = float(fix[f"{name}_eta"])
    for j, k in enumerate(kpoints_of(name)):
        d = dev.device(k)
        ll = tuple(fix[f"{name}_l_{key}"][j] for key in ("d00", "d01", "d10"))
        lr = tuple(fix[f"{name}_r_{key}"][j] for key in ("d00", "d01", "d10"))
        for i, w in enumerate(fix[f"{name}_omegas"]):
            t = transmission_point(float(w), list(d.onsite_blocks), list(d.coupling_blocks), ll, lr, eta=eta,
                                   vl=fix[f"{name}_vl"][j], vr=fix[f"{name}_vr"][j])
            ref = float(fix[f"{name}_T"][i, j])
            assert abs(t - ref) <= 1e-10 * max(1.0, abs(ref)), (name, i, k, t, ref)
