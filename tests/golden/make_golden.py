"""Generate the golden vectors of the NEGF path by running negfpy itself.

Run from the repository root and name negfpy's ``src`` directory, either with
``--ref`` or in the NEGFPY_SRC environment variable:

    python tests/golden/make_golden.py --ref /path/to/negfpy/src

Inputs are the seeded synthetic workloads of ``negfpy_b200.workloads`` (their
blocks are stored with the outputs, so the fixtures do not depend on the
generator staying bit-stable), plus the small analytic systems of negfpy's
own test-suite.  Every output here is computed by negfpy's public functions
(``transmission``, ``surface_gf``, ``lead_surface_dos``, the workflow's
``_thermal_conductance_from_spectrum``) in FP64 with Sancho-Rubio, and for a
few points also with the QEP eigen method as an independent cross-check.
"""

from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
OUT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))


def thermal(out_dir: Path) -> None:
    """thermal.npz: negfpy's heat currents (core/thermal_current.py) on chain and square-lattice spectra."""
    import negfpy.core as R
    from negfpy.models import ChainParams, SquareLatticeParams, device_perfect_chain, lead_blocks
    from negfpy.models import square_lattice_device, square_lattice_lead

    from negfpy_b200 import workloads as W

    wl = W.chain_workload()
    unit = wl.omega_unit_rad_s
    p = ChainParams(1.0, 1.0)
    lead = lead_blocks(p)
    dev = device_perfect_chain(8, p)
    t_chain = np.array([R.transmission(float(w), dev, lead, lead, eta=1e-8) for w in wl.omegas])
    om_rad = wl.omegas * unit
    pairs = np.array([[310.0, 290.0], [50.0, 40.0], [1000.0, 10.0], [300.0, 300.0]])
    j_spec = np.array([R.heat_current_from_spectrum(om_rad, t_chain, a, b) for a, b in pairs])
    # heat_current_1d: its omegas are passed to transmission as they are (model units) and also used as rad/s
    om1 = np.linspace(0.05, 1.95, 48)
    j1 = R.heat_current_1d(om1, device_perfect_chain(6, p), lead, lead, 1e-10, 0.5e-10, eta=1e-8)
    sq = SquareLatticeParams(mass=1.0, spring_x=1.0, spring_y=0.5)
    kp = [(-np.pi / 2,), (0.0,), (np.pi / 3,)]
    om2 = np.linspace(0.1, 2.2, 32)
    j2 = R.heat_current_per_length_2d(om2, square_lattice_device(5, sq), square_lattice_lead(sq), square_lattice_lead(sq),
                                      kp, 2.5, 2e-10, 1e-10, eta=1e-7)
    j3 = R.heat_current_density_3d(om2, square_lattice_device(5, sq), square_lattice_lead(sq), square_lattice_lead(sq),
                                   kp, 4.0, 2e-10, 1e-10, eta=1e-7)
    tl = R.transverse_length_from_vector([1.0, 2.0, 0.5], [0.0, 1.0, 0.0])
    # full counting statistics (core/fcs.py) on the chain spectrum and on k moments of the square lattice
    from negfpy.core import fcs as F

    c_spec = np.array([[F.heat_current_cumulants_from_spectrum(om_rad, t_chain, a, b).c1_j_per_s,
                        F.heat_current_cumulants_from_spectrum(om_rad, t_chain, a, b).c2_j2_per_s] for a, b in pairs])
    sqdev, sqlead = square_lattice_device(5, sq), square_lattice_lead(sq)
    t_wk = np.array([[R.transmission(float(w), sqdev, sqlead, sqlead, eta=1e-7, kpar=k) for k in kp] for w in om2])
    t1, t2 = t_wk.mean(axis=1), (t_wk ** 2).mean(axis=1)
    om2_rad = om2 * unit
    cm = F.heat_current_cumulants_from_k_moments(om2_rad, t1, t2, 300.0, 280.0)
    unc = F.heat_current_uncertainty(cm, measurement_time_s=1e-6)
    np.savez_compressed(out_dir / "thermal.npz", om_rad=om_rad, t_chain=t_chain, pairs=pairs, j_spec=j_spec,
                        om1=om1, j1=j1, om2=om2, kp=np.array(kp), j2=j2, j3=j3, tl=tl, c_spec=c_spec,
                        t_wk=t_wk, om2_rad=om2_rad, c_mom=np.array([cm.c1_j_per_s, cm.c2_j2_per_s]),
                        unc=np.array([unc.std_current_j_per_s, unc.variance_energy_j2, unc.std_energy_j]))


def green(out_dir: Path) -> None:
    """green.npz: negfpy's device_green_function (core/negf.py:253-303) on small systems."""
    import negfpy.core as R
    from negfpy.core.types import Device1D, LeadBlocks
    from negfpy.models import ChainParams, MultiDofCellParams, device_perfect_chain, lead_blocks
    from negfpy.models import multidof_device, multidof_lead_blocks

    from negfpy_b200 import workloads as W

    out = {}
    p = ChainParams(1.0, 1.0)
    lead = lead_blocks(p)
    out["chain_G"], out["chain_SL"], out["chain_SR"] = R.device_green_function(1.1, device_perfect_chain(6, p), lead,
                                                                               lead, eta=1e-8)
    lead1 = LeadBlocks(d00=np.array([[2.0]], dtype=np.complex128), d01=np.array([[-1.0]], dtype=np.complex128))
    onsite = [np.diag([2.0, 100.0]).astype(np.complex128) for _ in range(4)]
    coupling = [np.diag([-1.0, 0.0]).astype(np.complex128) for _ in range(3)]
    out["rect_G"], out["rect_SL"], out["rect_SR"] = R.device_green_function(
        1.0, Device1D(onsite, coupling), lead1, lead1, eta=1e-8, device_to_lead_left=np.array([[-1.0]]),
        device_to_lead_right=np.array([[-1.0]]), contact_left_indices=[0], contact_right_indices=[6])
    md = MultiDofCellParams(masses=np.ones(2), fc00=2.0 * np.eye(6), fc01=-np.eye(6), dof_per_atom=3)
    out["md_G"], out["md_SL"], out["md_SR"] = R.device_green_function(0.7, multidof_device(5, md),
                                                                      multidof_lead_blocks(md),
                                                                      multidof_lead_blocks(md), eta=1e-7,
                                                                      eta_device=2e-7)
    wl = W.slab_workload()
    ki = 13
    lb = LeadBlocks(d00=wl.lead_l["d00"][ki], d01=wl.lead_l["d01"][ki], d10=wl.lead_l["d10"][ki])
    dv = Device1D(onsite_blocks=[wl.onsite[ki, 0]] * 3, coupling_blocks=[wl.coupling[ki, 0]] * 2)
    out["slab_G"], out["slab_SL"], out["slab_SR"] = R.device_green_function(float(wl.omegas[900]), dv, lb, lb,
                                                                            eta=wl.eta, omega_scale=1.3)
    out["slab_omega"], out["slab_eta"], out["slab_k"] = float(wl.omegas[900]), wl.eta, ki
    np.savez_compressed(out_dir / "green.npz", **out)


WORKFLOW_OMEGAS = [-0.1, 0.0, 0.3, 0.7, 1.1, 1.8, 2.5, 3.3]
WORKFLOW_KMESH = {"low_cm1": 1e5, "low": {"kpoints": [(0.0,), (1.2,)]}, "high": {"kpoints": [(-2.0,), (0.4,), (2.6,)]}}
WORKFLOW_CFGS = {
    "adaptive": {"solver": {"surface_gf_method": "sancho_rubio", "eta_scheme": "adaptive",
                            "eta_values": [1e-7, 1e-5, 1e-3], "max_channel_factor": 0.15,
                            "min_success_fraction": 0.3, "collect_rejected": True}},
    "global": {"solver": {"surface_gf_method": "sancho_rubio", "eta_scheme": "adaptive-global",
                          "eta_values": [1e-7, 1e-5, 1e-3], "max_channel_factor": 0.2,
                          "min_success_fraction": 0.6, "collect_rejected": True, "max_eta_over_omega": 1e-4,
                          "eta_ratio_cm1_min": 5e4, "eta_device": 2e-6}},
    "fixed": {"solver": {"surface_gf_method": "sancho_rubio", "eta_scheme": "fixed", "eta_fixed": 3e-6,
                         "omega_scale_mode": "ev", "parallel": {"enabled": True, "workers": 4}}},
    "strict": {"solver": {"surface_gf_method": "sancho_rubio", "eta_scheme": "adaptive", "eta_values": [1e-7, 1e-5],
                          "max_channel_factor": 0.08, "min_success_fraction": 1.0}},
    "strict_global": {"solver": {"surface_gf_method": "sancho_rubio", "eta_scheme": "adaptive_global",
                                 "eta_values": [1e-7, 1e-5], "max_channel_factor": 0.08,
                                 "min_success_fraction": 1.0, "collect_rejected": True}},
}


def workflow_system(params_cls, lead_fn, dev_fn):
    """The small slab of the workflow fixture (seeded spring network, 4 layers)."""
    from negfpy_b200 import workloads as W

    p = W.spring_network(2, ny=2, nz=8, periodic_y=True, periodic_z=False)
    prm = params_cls(masses=p.masses, fc00_terms=p.fc00_terms, fc01_terms=p.fc01_terms, dof_per_atom=3)
    return dev_fn(4, prm), lead_fn(prm)


def workflow(out_dir: Path) -> None:
    """workflow.npz: negfpy's _run_transmission (workflows/ifc_bulk.py:1059-1288) on a small slab."""
    import json

    from negfpy.models.material_kspace import MaterialKspaceParams, material_kspace_device, material_kspace_lead
    from negfpy.workflows import ifc_bulk

    dev, lead = workflow_system(MaterialKspaceParams, material_kspace_lead, material_kspace_device)
    out = {}
    for name, cfg in WORKFLOW_CFGS.items():
        res = ifc_bulk._run_transmission(cfg, device=dev, lead_left=lead, lead_right=lead,
                                         omegas=np.array(WORKFLOW_OMEGAS), kmesh=WORKFLOW_KMESH)
        out[name + "_values"] = res["values"]
        meta = {k: res[k] for k in ("eta_records", "omega_failures", "n_rejected_total", "summary")}
        out[name + "_meta"] = np.array(json.dumps(meta, default=lambda o: list(o) if isinstance(o, tuple) else o))
    np.savez_compressed(out_dir / "workflow.npz", **out)


INTERFACE_KPOINTS = {"slab": [(-2.7,), (-0.4,), (0.0,), (1.3,), (3.0,)],
                     "bulk": [(0.0, 0.0), (0.7, -1.9), (-2.2, 2.9)]}
INTERFACE_LAYERS = {"slab": 4, "bulk": 3}
INTERFACE_FRACTIONS = (0.13, 0.41, 0.77)  # omega / omega_max of the T points


def interface_params(name: str, params_cls):
    """Seeded force-constant sets of the interface fixture: ``slab`` (n = 48,
    1D k, fc10 implied by fc01) and ``bulk`` (n = 12, 2D k, explicit fc10
    terms and an onsite pinning)."""
    from negfpy_b200 import workloads as W

    if name == "slab":
        p = W.spring_network(2, ny=2, nz=8, periodic_y=True, periodic_z=False)
        return params_cls(masses=p.masses, fc00_terms=p.fc00_terms, fc01_terms=p.fc01_terms, dof_per_atom=3)
    p = W.spring_network(3, ny=2, nz=2, periodic_y=True, periodic_z=True)
    fc10 = {(-dy, -dz): np.asarray(v).T.copy() for (dy, dz), v in p.fc01_terms.items()}
    return params_cls(masses=p.masses, fc00_terms=p.fc00_terms, fc01_terms=p.fc01_terms, fc10_terms=fc10,
                      dof_per_atom=3, onsite_pinning=0.02)


def _terms_arrays(prefix: str, terms) -> dict:
    if terms is None:
        return {}
    keys = list(terms.keys())
    return {prefix + "_keys": np.array(keys, dtype=np.int64), prefix + "_blocks": np.stack([terms[k] for k in keys])}


def interface(out_dir: Path) -> None:
    """interface.npz: negfpy's _build_interface_contacts (workflows/ifc_bulk.py:690-742),
    transmission through it, and _run_transmission on the slab set-up."""
    import json

    import negfpy.core as R
    from negfpy.models.material_kspace import MaterialKspaceParams, material_kspace_device
    from negfpy.workflows import ifc_bulk

    from negfpy_b200 import workloads as W

    out = {}
    for name in ("slab", "bulk"):
        prm = interface_params(name, MaterialKspaceParams)
        ll, lr, vdl_l, vdl_r = ifc_bulk._build_interface_contacts(prm)
        kp = INTERFACE_KPOINTS[name]
        blocks = {"l": [ll.blocks(k) for k in kp], "r": [lr.blocks(k) for k in kp]}
        for side in ("l", "r"):
            for i, key in enumerate(("d00", "d01", "d10")):
                out[f"{name}_{side}_{key}"] = np.stack([b[i] for b in blocks[side]])
        out[f"{name}_vl"] = np.stack([vdl_l(k) for k in kp])
        out[f"{name}_vr"] = np.stack([vdl_r(k) for k in kp])
        out[f"{name}_masses"] = np.asarray(prm.masses, dtype=float)
        out[f"{name}_pinning"] = float(prm.onsite_pinning)
        out.update(_terms_arrays(f"{name}_fc00", prm.fc00_terms))
        out.update(_terms_arrays(f"{name}_fc01", prm.fc01_terms))
        out.update(_terms_arrays(f"{name}_fc10", prm.fc10_terms))
        wmax = W.estimate_omega_max(prm, nk=6, two_d=(name == "bulk"))
        eta = 1e-5 * wmax * wmax
        dev = material_kspace_device(n_layers=INTERFACE_LAYERS[name], params=prm)
        om = np.array([f * wmax for f in INTERFACE_FRACTIONS])
        out[f"{name}_omegas"] = om
        out[f"{name}_eta"] = eta
        out[f"{name}_T"] = np.array([[R.transmission(float(w), dev, ll, lr, eta=eta, kpar=k, device_to_lead_left=vdl_l,
                                                     device_to_lead_right=vdl_r) for k in kp] for w in om])
    prm = interface_params("slab", MaterialKspaceParams)
    ll, lr, vdl_l, vdl_r = ifc_bulk._build_interface_contacts(prm)
    dev = material_kspace_device(n_layers=4, params=prm)
    # the per-omega k averages and eta ladders through the same contacts
    kp = INTERFACE_KPOINTS["slab"]
    w = float(out["slab_omegas"][1])
    wmax2 = (w / INTERFACE_FRACTIONS[1]) ** 2
    kw = dict(device_to_lead_left=vdl_l, device_to_lead_right=vdl_r)
    ladder = tuple(f * wmax2 for f in (1e-7, 1e-5, 1e-3))
    out["kavg"] = R.transmission_kavg(w, dev, ll, lr, kpoints=kp, eta=float(out["slab_eta"]), **kw)
    val, info = R.transmission_kavg_adaptive(w, dev, ll, lr, kpoints=kp, eta_values=ladder, max_channel_factor=0.2,
                                             collect_rejected=True, **kw)
    out["adaptive_value"], out["adaptive_info"] = val, np.array(json.dumps(info, default=list))
    val, info = R.transmission_kavg_adaptive_global_eta(w, dev, ll, lr, kpoints=kp, eta_values=ladder,
                                                        max_channel_factor=0.2, min_success_fraction=0.3,
                                                        collect_rejected=True, **kw)
    out["global_value"], out["global_info"] = val, np.array(json.dumps(info, default=list))
    out["ladder"] = np.array(ladder)
    res = ifc_bulk._run_transmission(WORKFLOW_CFGS["adaptive"], device=dev, lead_left=ll, lead_right=lr,
                                     device_to_lead_left=vdl_l, device_to_lead_right=vdl_r,
                                     omegas=np.array(WORKFLOW_OMEGAS), kmesh=WORKFLOW_KMESH)
    out["workflow_values"] = res["values"]
    meta = {k: res[k] for k in ("eta_records", "omega_failures", "n_rejected_total", "summary")}
    out["workflow_meta"] = np.array(json.dumps(meta, default=lambda o: list(o) if isinstance(o, tuple) else o))
    np.savez_compressed(out_dir / "interface.npz", **out)


DOS_KPOINTS = [(0.0, 0.0), (1.1, -0.6), (-2.5, 2.2), (2.9, 0.4)]


def poisoned_blocks(lead, k):
    """The lead's blocks, with NaN everywhere at the last k point of DOS_KPOINTS."""
    d00, d01, d10 = (np.array(b, dtype=complex) for b in lead.blocks(k))
    if tuple(k) == DOS_KPOINTS[-1]:
        d00 = np.full_like(d00, np.nan)
    return d00, d01, d10


def dos(out_dir: Path) -> None:
    """dos.npz: negfpy's k-averaged, adaptive and spectrum forms of the lead
    surface DOS (core/dos.py:64-252) on a 2D-k material lead (n = 12) and on
    the two different leads of its interface contacts."""
    import json

    import negfpy.core.dos as D
    from negfpy.models.material_kspace import MaterialKspaceParams, material_kspace_lead
    from negfpy.workflows import ifc_bulk

    from negfpy_b200 import workloads as W

    from negfpy.core.types import LeadKSpace

    prm = interface_params("bulk", MaterialKspaceParams)
    lead = material_kspace_lead(prm)
    ll, lr, _, _ = ifc_bulk._build_interface_contacts(prm)
    wmax = W.estimate_omega_max(prm, nk=6, two_d=True)
    eta = 1e-5 * wmax * wmax
    om = np.array([0.17, 0.45, 0.83]) * wmax
    # The ladder's failure path, made deterministic: the last k point has NaN
    # blocks, so it fails at every eta and counts as failed.
    ladder = (1e-5 * wmax * wmax, 1e-3 * wmax * wmax)
    poisoned = LeadKSpace(blocks_builder=lambda k: poisoned_blocks(lead, k))
    out = {"omegas": om, "eta": eta, "ladder": np.array(ladder)}
    out["kavg"] = np.array([D.lead_surface_dos_kavg(float(w), lead, DOS_KPOINTS, eta) for w in om])
    out["kavg_norm"] = np.array([D.lead_surface_dos_kavg(float(w), lead, DOS_KPOINTS, eta, normalize_per_mode=True)
                                 for w in om])
    vals, infos = [], []
    for w in om:
        v, info = D.lead_surface_dos_kavg_adaptive(float(w), poisoned, DOS_KPOINTS, ladder, 0.5)
        vals.append(v)
        infos.append(info)
    out["adaptive"] = np.array(vals)
    out["adaptive_info"] = np.array(json.dumps(infos))
    out["spectrum_k"] = D.lead_surface_dos_spectrum(om, lead, kpoints=DOS_KPOINTS, eta=eta)
    out["spectrum_ladder"] = D.lead_surface_dos_spectrum(om, poisoned, kpoints=DOS_KPOINTS, eta_values=ladder,
                                                         min_success_fraction=0.5)
    out["spectrum_gamma"] = D.lead_surface_dos_spectrum(om, lead, eta=eta)
    two = D.leads_surface_dos_spectrum(om, ll, lr, kpoints=DOS_KPOINTS, eta=eta, normalize_per_mode=True)
    out["leads_left"], out["leads_right"] = two["left"], two["right"]
    np.savez_compressed(out_dir / "dos.npz", **out)


# negfpy's own study runs of real materials: (fixture name, run directory
# under negfpy's studies/).  Each run directory holds the configuration the
# run used (input.json), the transmission it wrote (transmission.tsv) and its
# eta records (transmission_eta_diag.json).
STUDY_RUNS = [
    ("silicon_x", "silicon_bulk_2026q1/silicon/runs/20260225_033931Z_silicon_transmission_x"),
    ("tan_x", "TaN/TaN/runs/20260225_113114Z_tan_transmission_x"),
    ("graphene", "graphene_bulk_2026q1/graphene/runs/20260226_033848Z_graphene_transmission"),
    ("phosphorene_x", "phosphorene_p_zerostrain_2026q1/phosphorene_p_zerostrain/runs/"
                      "20260226_032511Z_phosphorene_p_zerostrain_transmission_x_area"),
    ("borophene_y", "borophene_b_2x1_pbe_2026q1/borophene_b_2x1_pbe/runs/"
                    "20260225_033229Z_borophene_b_2x1_pbe_transmission_y"),
    ("stanene_y", "stanene_1l_orthogonal_2026q1/stanene_1l_orthogonal/runs/"
                  "20260226_031515Z_stanene_1l_orthogonal_transmission_y_area"),
    ("beta12_x", "borophene_b_beta12_2026q1/borophene_b_beta12/runs/"
                 "20260226_034715Z_borophene_b_beta12_transmission_area"),
    ("beta12_y", "borophene_b_beta12_2026q1/borophene_b_beta12/runs/"
                 "20260226_035209Z_borophene_b_beta12_transmission_area_y"),
]


# negfpy's thermal-conductance study runs: (fixture name, run directory).
# Each turns the transmission.tsv of a transmission run into G(T) with the
# workflow's _thermal_conductance_from_spectrum (workflows/ifc_bulk.py:408-438).
THERMAL_RUNS = [
    ("tan_x", "TaN/TaN/runs/20260225_120308Z_tan_thermal_x"),
    ("silicon_x", "silicon_bulk_2026q1/silicon/runs/20260226_034402Z_silicon_thermal_x_area"),
    ("graphene_x", "graphene_bulk_2026q1/graphene/runs/20260226_034402Z_graphene_thermal_x_area"),
    ("borophene_y", "borophene_b_2x1_pbe_2026q1/borophene_b_2x1_pbe/runs/"
                    "20260225_085015Z_borophene_b_2x1_pbe_thermal_y"),
]


def thermal_source(run_dir: Path) -> Path:
    """The transmission.tsv a thermal run read (workflows/ifc_bulk.py:1444-1468)."""
    import json

    cfg = json.loads((run_dir / "input.json").read_text())
    report = run_dir.parents[2] / "inputs" / "configs" / cfg["thermal"]["transmission_report_path"]
    return report.resolve().parent / "transmission.tsv"


def study_setup(run_dir: Path, ifc_path: str | None = None):
    """The inputs negfpy's run_ifc_bulk hands to _run_transmission (or
    _run_fcs) for one study run (workflows/ifc_bulk.py:2186-2296): IFC read,
    reoriented and cut, the material parameters with their mass mode and
    transverse controls, the device layer count, the k meshes and the omega
    grid.  ``ifc_path`` replaces a force-constant path that only existed on
    the machine of the run, relative to the study's inputs/configs."""
    import json

    from negfpy.workflows import ifc_bulk as IB

    cfg = json.loads((run_dir / "input.json").read_text())
    cfg_dir = run_dir.parents[2] / "inputs" / "configs"
    icfg, mcfg = dict(cfg.get("ifc", {})), dict(cfg.get("model", {}))
    if ifc_path is not None:
        icfg["path"] = ifc_path
    ifc = IB.read_ifc(IB._resolve_path(cfg_dir, icfg.get("path", "si444.fc")), reader=str(icfg.get("reader", "qe")))
    if bool(icfg.get("enforce_asr", False)):
        ifc, _ = IB.enforce_translational_asr_on_self_term(ifc)
    ifc = IB._reorient_ifc_for_transport_direction(ifc, direction=int(mcfg.get("transport_direction", 1)))
    cut = lambda key: None if icfg.get(key) is None else int(icfg[key])  # noqa: E731
    ifc, _ = IB._apply_transverse_cutoff(ifc, dy_cutoff=cut("dy_cutoff"), dz_cutoff=cut("dz_cutoff"))
    pls = mcfg.get("principal_layer_size", None)
    bc = IB.BuildConfig(onsite_pinning=float(mcfg.get("onsite_pinning", 0.0)),
                        principal_layer_size=None if pls is None else int(pls),
                        auto_principal_layer_enlargement=bool(mcfg.get("auto_principal_layer_enlargement", True)),
                        infer_fc01_from_negative_dx=bool(mcfg.get("infer_fc01_from_negative_dx", True)),
                        enforce_hermitian_fc00=bool(mcfg.get("enforce_hermitian_fc00", True)),
                        nyquist_split_half=bool(mcfg.get("nyquist_split_half", False)),
                        dtype=str(mcfg.get("dtype", "complex128")))
    prm = IB.build_material_kspace_params(ifc=ifc, config=bc)
    prm, _ = IB._apply_mass_mode(prm, mcfg.get("mass_mode", "ifc"))
    prm, _, _ = IB._apply_transverse_stability_controls(prm, ifc_metadata=dict(ifc.metadata),
                                                        drop_nyquist=bool(mcfg.get("drop_nyquist_transverse", False)))
    omegas, _ = IB._build_omega_grid(cfg, ifc)
    if ifc_path is None:
        return cfg, prm, int(mcfg.get("n_layers", 30)), IB._prepare_kmesh(cfg), omegas
    thick, tdir, lvo = (mcfg.get(k, None) for k in ("thickness_angstrom", "thickness_direction",
                                                    "lattice_vectors_angstrom"))
    lv = IB._resolve_lattice_vectors_for_area(
        ifc_lattice_vectors=None if ifc.lattice_vectors is None else np.asarray(ifc.lattice_vectors, dtype=float),
        ifc_metadata=dict(ifc.metadata),
        lattice_vectors_override_angstrom=None if lvo is None else np.asarray(lvo, dtype=float))
    area = IB._compute_effective_area_m2(lv, transport_direction=int(mcfg.get("transport_direction", 1)),
                                         thickness_m=None if thick is None else float(thick) * IB.ANGSTROM_M,
                                         thickness_direction=None if tdir is None else int(tdir))
    return cfg, prm, int(mcfg.get("n_layers", 30)), IB._prepare_kmesh(cfg), omegas, float(area)


def _real_if_real(a):
    a = np.asarray(a)
    return a.real.copy() if np.iscomplexobj(a) and not np.any(a.imag) else a


def studies(out_dir: Path, studies_root: Path) -> None:
    """studies.npz: the material parameters, meshes and grids of negfpy's study
    runs (study_setup), with the transmission and eta records those runs
    wrote (negfpy's output files, computed with the QEP surface GF), and the
    same workflow stage re-run here by negfpy with Sancho-Rubio (``sr_*``)."""
    import json

    from negfpy.workflows import ifc_bulk as IB

    out = {}
    for name, rel in STUDY_RUNS:
        run = studies_root / rel
        cfg, prm, n_layers, kmesh, omegas = study_setup(run)
        ll, lr, vdl_l, vdl_r = IB._build_interface_contacts(prm)
        dev = IB.material_kspace_device(n_layers=n_layers, params=prm)
        sr_cfg = json.loads(json.dumps(cfg))
        sr_cfg["solver"]["surface_gf_method"] = "sancho_rubio"
        sr_cfg["solver"]["parallel"] = {"enabled": True, "backend": "process", "workers": os.cpu_count() or 1}
        res = IB._run_transmission(sr_cfg, device=dev, lead_left=ll, lead_right=lr, device_to_lead_left=vdl_l,
                                   device_to_lead_right=vdl_r, omegas=omegas, kmesh=kmesh)
        out[f"{name}_sr_values"] = np.asarray(res["values"], dtype=float)
        meta = {k: res[k] for k in ("eta_records", "omega_failures", "n_rejected_total")}
        out[f"{name}_sr_meta"] = np.array(json.dumps(meta, default=lambda o: list(o) if isinstance(o, tuple) else o))
        tsv = np.loadtxt(run / "transmission.tsv")
        assert np.abs(tsv[:, 0] - omegas).max() <= 1e-12 * max(1.0, float(np.abs(omegas).max())), name
        diag = json.loads((run / "transmission_eta_diag.json").read_text())
        out[f"{name}_cfg"] = np.array(json.dumps(cfg))
        out[f"{name}_kmesh"] = np.array(json.dumps(kmesh, default=list))
        out[f"{name}_omegas"] = np.asarray(omegas, dtype=float)
        out[f"{name}_n_layers"] = n_layers
        out[f"{name}_T"] = tsv[:, 3].copy()
        out[f"{name}_diag"] = np.array(json.dumps(diag))
        out[f"{name}_masses"] = np.asarray(prm.masses, dtype=float)
        out[f"{name}_pinning"] = float(prm.onsite_pinning)
        out[f"{name}_dof"] = int(prm.dof_per_atom)
        for key in ("fc00", "fc01", "fc10"):
            terms = getattr(prm, key + "_terms")
            if terms is not None:
                out.update(_terms_arrays(f"{name}_{key}", {k: _real_if_real(v) for k, v in terms.items()}))
    for name, rel in THERMAL_RUNS:
        run = studies_root / rel
        src = np.loadtxt(thermal_source(run))
        tab = np.loadtxt(run / "thermal_conductance.tsv")
        out[f"thermal_{name}_spectrum"] = src  # omega_qe, THz, cm^-1, T[, T per m^2]
        out[f"thermal_{name}_table"] = tab  # temperature, G, G per m^2
    np.savez_compressed(out_dir / "studies.npz", **out)


FCS_STUDY_RUN = "TaN/TaN/runs/20260304_104756Z_tan_x_fcs_cond_area_20260304"
FCS_STUDY_IFC = "../../FORCE_CONSTANTS"  # the run's own path pointed at its author's machine
# Configuration variants of the FCS stage on the silicon study's material, on
# a 16/36-point k mesh: every x/y mode, the three temperature sweeps and the
# fixed and global eta schemes.
FCS_KMESH_CFG = {"dimension": 2, "mode": "shifted", "nk": 4, "nk_low": 6, "low_cm1": 120.0}
FCS_CFGS = {
    "delta_conductance": {
        "solver": {"surface_gf_method": "sancho_rubio", "eta_scheme": "adaptive_global",
                   "eta_values": [1e-8, 1e-6, 1e-4], "min_success_fraction": 0.7},
        "fcs": {"x": "temperature", "y": "conductance", "temperature_mode": "fixed_delta", "delta_t_k": 5.0,
                "temperature_min_k": 10.0, "temperature_max_k": 500.0, "n_points": 25}},
    "right_heat_current": {
        "solver": {"surface_gf_method": "sancho_rubio", "eta_scheme": "fixed", "eta_fixed": 1e-6},
        "fcs": {"x": "temperature", "y": "heat_current", "temperature_mode": "fixed_right",
                "temperature_right_k": 200.0, "temperature_min_k": 5.0, "temperature_max_k": 800.0, "n_points": 17,
                "measurement_time_s": 3e-9}},
    "bias_per_area": {
        "solver": {"surface_gf_method": "sancho_rubio", "eta_scheme": "adaptive", "eta_values": [1e-8, 1e-7, 1e-5],
                   "min_success_fraction": 1.0, "max_eta_over_omega": 2e-4, "eta_ratio_cm1_min": 50.0,
                   "nonnegative_tolerance": 1e-12},
        "fcs": {"x": "temperature_bias", "y": "heat_current_per_area", "temperature_avg_k": 300.0,
                "temperature_min_k": -100.0, "temperature_max_k": 100.0, "n_points": 21}},
}
FCS_KEYS = ("t_mean", "t2_mean", "eta_selected", "n_k_success", "x", "temp_left_k", "temp_right_k", "y", "y_std",
            "c1_j_per_s", "c2_j2_per_s")


def fcs(out_dir: Path, studies_root: Path) -> None:
    """fcs.npz: negfpy's FCS stage (_run_fcs, workflows/ifc_bulk.py:1690-1935)
    with Sancho-Rubio on the silicon study's material for the FCS_CFGS
    variants, and on the TaN FCS study run's inputs, whose own outputs
    (fcs_moments.npz and fcs.tsv, written with the QEP surface GF) are stored
    beside it as ``tan_pub_*``."""
    import json

    from negfpy.workflows import ifc_bulk as IB

    out = {}

    def run(prefix, cfg, prm, n_layers, kmesh, omegas, area):
        ll, lr, vdl_l, vdl_r = IB._build_interface_contacts(prm)
        dev = IB.material_kspace_device(n_layers=n_layers, params=prm)
        res = IB._run_fcs(cfg, omegas=omegas, kmesh=kmesh, device=dev, lead_left=ll, lead_right=lr,
                          device_to_lead_left=vdl_l, device_to_lead_right=vdl_r, area_m2=area)
        for key in FCS_KEYS:
            out[f"{prefix}_{key}"] = np.asarray(res[key])
        out[f"{prefix}_failures"] = np.array(json.dumps(res["omega_failures"]))

    def store_params(prefix, prm):
        out[f"{prefix}_masses"] = np.asarray(prm.masses, dtype=float)
        out[f"{prefix}_pinning"] = float(prm.onsite_pinning)
        out[f"{prefix}_dof"] = int(prm.dof_per_atom)
        for key in ("fc00", "fc01", "fc10"):
            terms = getattr(prm, key + "_terms")
            if terms is not None:
                out.update(_terms_arrays(f"{prefix}_{key}", {k: _real_if_real(v) for k, v in terms.items()}))

    si_run = studies_root / dict(STUDY_RUNS)["silicon_x"]
    _, si_prm, si_layers, _, si_om = study_setup(si_run)
    km = IB._prepare_kmesh({"kmesh": FCS_KMESH_CFG})
    out["si_kmesh"] = np.array(json.dumps(km, default=list))
    out["si_omegas"], out["si_n_layers"], out["si_area"] = si_om, si_layers, 3.1e-19
    store_params("si", si_prm)
    for name, cfg in FCS_CFGS.items():
        run(name, cfg, si_prm, si_layers, km, si_om, 3.1e-19)

    tan_run = studies_root / FCS_STUDY_RUN
    cfg, prm, n_layers, kmesh, omegas, area = study_setup(tan_run, FCS_STUDY_IFC)
    cfg["ifc"]["path"] = FCS_STUDY_IFC
    out["tan_cfg"] = np.array(json.dumps(cfg))
    out["tan_kmesh"] = np.array(json.dumps(kmesh, default=list))
    out["tan_omegas"], out["tan_n_layers"], out["tan_area"] = omegas, n_layers, area
    store_params("tan", prm)
    pub = np.load(tan_run / "fcs_moments.npz")
    assert np.abs(pub["omega_qe"] - omegas).max() <= 1e-12 * float(np.abs(omegas).max())
    for key in ("t_mean", "t2_mean", "eta_selected", "n_k_success"):
        out[f"tan_pub_{key}"] = pub[key]
    out["tan_pub_table"] = np.loadtxt(tan_run / "fcs.tsv")
    sr_cfg = json.loads(json.dumps(cfg))
    sr_cfg["solver"]["surface_gf_method"] = "sancho_rubio"
    run("tan_sr", sr_cfg, prm, n_layers, kmesh, omegas, area)
    np.savez_compressed(out_dir / "fcs.npz", **out)


# Configuration variants of the workflow's DOS stage on the right interface
# lead of the silicon study's material (n = 12, the FCS k mesh), with a
# negative omega; the "nan_*" variants poison one k point of the high mesh.
# The study grid's omega = 0 is left out: there z = -eta^2 is real, and
# whether the decimation converges or overflows at a k point depends on
# rounding (as for eta = 0 at any omega).
DOS_WORKFLOW_CFGS = {
    "fixed": {"solver": {"surface_gf_method": "sancho_rubio", "eta_scheme": "fixed", "eta_fixed": 1e-6},
              "dos": {"normalize_per_mode": True}},
    "global": {"solver": {"surface_gf_method": "sancho_rubio", "eta_scheme": "adaptive_global",
                          "eta_values": [1e-8, 1e-6, 1e-4], "min_success_fraction": 0.7, "max_eta_over_omega": 2e-3,
                          "eta_ratio_cm1_min": 60.0}, "dos": {"negative_tolerance": 1e-10}},
    "per_k": {"solver": {"surface_gf_method": "sancho_rubio", "eta_scheme": "adaptive", "eta_values": [1e-8, 1e-7],
                         "min_success_fraction": 0.5}},
    "nan_fixed": {"solver": {"surface_gf_method": "sancho_rubio", "eta_scheme": "fixed", "eta_fixed": 1e-6}},
    "nan_global": {"solver": {"surface_gf_method": "sancho_rubio", "eta_scheme": "adaptive-global",
                              "eta_values": [1e-8, 1e-6], "min_success_fraction": 0.9}},
    "nan_per_k": {"solver": {"surface_gf_method": "sancho_rubio", "eta_scheme": "adaptive",
                             "eta_values": [1e-8, 1e-6], "min_success_fraction": 0.95}},
}
DOS_NAN_K = 2  # index into the high k mesh


def nan_at(lead, kbad):
    """The lead's blocks, with NaN everywhere at k point ``kbad``."""
    def blocks(k):
        d00, d01, d10 = (np.array(b, dtype=complex) for b in lead.blocks(k))
        if tuple(k) == tuple(kbad):
            d00 = np.full_like(d00, np.nan)
        return d00, d01, d10
    return blocks


def dos_workflow(out_dir: Path, studies_root: Path) -> None:
    """dos_workflow.npz: negfpy's _run_dos (workflows/ifc_bulk.py:1290-1441)
    with Sancho-Rubio for the DOS_WORKFLOW_CFGS variants."""
    import json

    from negfpy.core.types import LeadKSpace
    from negfpy.workflows import ifc_bulk as IB

    _, prm, _, _, om = study_setup(studies_root / dict(STUDY_RUNS)["silicon_x"])
    km = IB._prepare_kmesh({"kmesh": FCS_KMESH_CFG})
    omegas = np.concatenate([[-1e-4], om[1:]])
    _, lead, _, _ = IB._build_interface_contacts(prm)
    bad = LeadKSpace(blocks_builder=nan_at(lead, km["high"]["kpoints"][DOS_NAN_K]))
    out = {"omegas": omegas, "kmesh": np.array(json.dumps(km, default=list))}
    for name, cfg in DOS_WORKFLOW_CFGS.items():
        res = IB._run_dos(cfg, lead=bad if name.startswith("nan") else lead, omegas=omegas, kmesh=km)
        out[f"{name}_values"] = res["values"]
        meta = {k: res[k] for k in ("eta_records", "omega_failures", "summary")}
        out[f"{name}_meta"] = np.array(json.dumps(meta, default=lambda o: list(o) if isinstance(o, tuple) else o))
    # negfpy's messages for a decimation that overflows from finite blocks and
    # for NaN blocks, at the orders of the three kernel families
    from negfpy.core import surface_gf

    msgs = {}
    for n in SR_FAILURE_ORDERS:
        for case, (d00, d01) in sr_failure_blocks(n).items():
            try:
                surface_gf(0.5, d00, d01, eta=1e-8, method="sancho_rubio")
                msgs[f"{case}_{n}"] = None
            except Exception as exc:  # the message is the fixture
                msgs[f"{case}_{n}"] = f"{type(exc).__name__}: {exc}"
    out["sr_failure_messages"] = np.array(json.dumps(msgs))
    np.savez_compressed(out_dir / "dos_workflow.npz", **out)


SR_FAILURE_ORDERS = (1, 4, 64)


def sr_failure_blocks(n: int) -> dict:
    """Lead blocks whose decimation fails: coupling 1e200 (the first
    iteration's products overflow from finite blocks) and NaN blocks."""
    eye = np.eye(n, dtype=complex)
    return {"overflow": (eye, 1e200 * eye), "nan": (np.full((n, n), np.nan, dtype=complex), eye)}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("NEGFPY_SRC"),
                    help="negfpy's src directory (default: $NEGFPY_SRC)")
    ap.add_argument("--only", choices=["thermal", "green", "workflow", "interface", "dos", "studies", "fcs", "dos_workflow"], default=None,
                    help="write one fixture file only")
    args = ap.parse_args()
    if not args.ref:
        ap.error("name negfpy's src directory with --ref or NEGFPY_SRC")
    sys.path.insert(0, args.ref)
    if args.only == "thermal":
        thermal(OUT)
        print("wrote thermal.npz")
        return
    if args.only == "green":
        green(OUT)
        print("wrote green.npz")
        return
    if args.only == "workflow":
        workflow(OUT)
        print("wrote workflow.npz")
        return
    if args.only == "interface":
        interface(OUT)
        print("wrote interface.npz")
        return
    if args.only == "dos":
        dos(OUT)
        print("wrote dos.npz")
        return
    studies_root = Path(args.ref).resolve().parent / "studies"
    if args.only == "studies":
        studies(OUT, studies_root)
        print("wrote studies.npz")
        return
    if args.only == "fcs":
        fcs(OUT, studies_root)
        print("wrote fcs.npz")
        return
    if args.only == "dos_workflow":
        dos_workflow(OUT, studies_root)
        print("wrote dos_workflow.npz")
        return
    import negfpy.core as R
    from negfpy.core.types import Device1D, LeadBlocks
    from negfpy.models import (ChainParams, MultiDofCellParams, SquareLatticeParams, device_perfect_chain,
                               lead_blocks, multidof_device, multidof_lead_blocks, square_lattice_device,
                               square_lattice_lead)
    from negfpy.modeling.units import qe_omega_to_rad_s
    from negfpy.workflows.ifc_bulk import _thermal_conductance_from_spectrum

    from negfpy_b200 import workloads as W

    qe_unit = float(qe_omega_to_rad_s(1.0))

    # ---- chain: 1000 omega in (0, 2), L = 8, eta = 1e-8 --------------------
    wl = W.chain_workload()
    p = ChainParams(1.0, 1.0)
    lead = lead_blocks(p)
    dev = device_perfect_chain(8, p)
    t_chain = np.array([R.transmission(float(w), dev, lead, lead, eta=1e-8) for w in wl.omegas])
    g_chain = np.array([R.surface_gf(float(w), lead.d00, lead.d01, eta=1e-8)[0, 0] for w in wl.omegas[::50]])
    dos_chain = np.array([R.lead_surface_dos(float(w), lead, eta=1e-8) for w in wl.omegas[::50]])
    temps = np.array([50.0, 300.0, 1000.0])
    kappa_chain = _thermal_conductance_from_spectrum(wl.omegas * wl.omega_unit_rad_s / qe_unit, t_chain, temps)
    np.savez_compressed(OUT / "chain.npz", omegas=wl.omegas, T=t_chain, g_omegas=wl.omegas[::50], g=g_chain,
                        dos=dos_chain, temps=temps, kappa=kappa_chain, omega_unit_rad_s=wl.omega_unit_rad_s,
                        n_layers=8, eta=1e-8)

    # ---- slab (n = 48): a stratified subsample of the 2048 x 64 grid -------
    wl = W.slab_workload()
    wsel = np.array([40, 300, 600, 900, 1200, 1500, 1800, 1950, 2047])
    ksel = np.array([0, 13, 31, 50])
    pairs, t_slab = [], []
    lead_at = {}
    for ki in ksel:
        lead_at[ki] = LeadBlocks(d00=wl.lead_l["d00"][ki], d01=wl.lead_l["d01"][ki], d10=wl.lead_l["d10"][ki])
    for wi in wsel:
        for ki in ksel:
            dv = Device1D(onsite_blocks=[wl.onsite[ki, 0]] * wl.n_layers,
                          coupling_blocks=[wl.coupling[ki, 0]] * (wl.n_layers - 1))
            t_slab.append(R.transmission(float(wl.omegas[wi]), dv, lead_at[ki], lead_at[ki], eta=wl.eta))
            pairs.append((wi, ki))
    g_pts = [(600, 13), (1800, 50)]
    g_slab = np.stack([R.surface_gf(float(wl.omegas[wi]), lead_at[ki].d00, lead_at[ki].d01, lead_at[ki].d10,
                                    eta=wl.eta) for wi, ki in g_pts])
    g_slab_qep = np.stack([R.surface_gf(float(wl.omegas[wi]), lead_at[ki].d00, lead_at[ki].d01, lead_at[ki].d10,
                                        eta=wl.eta, method="generalized_eigen") for wi, ki in g_pts])
    dos_slab = np.array([R.lead_surface_dos(float(wl.omegas[wi]), lead_at[ki], eta=wl.eta) for wi, ki in pairs])
    np.savez_compressed(OUT / "slab.npz", omegas=wl.omegas[wsel], wsel=wsel, ksel=ksel,
                        kpoints=np.array([wl.kpoints[k] for k in ksel]), pairs=np.array(pairs), T=np.array(t_slab),
                        d00=wl.lead_l["d00"][ksel], d01=wl.lead_l["d01"][ksel], d10=wl.lead_l["d10"][ksel],
                        onsite=wl.onsite[ksel, 0], coupling=wl.coupling[ksel, 0], n_layers=wl.n_layers,
                        eta=wl.eta, omega_max=wl.omega_max, g_pts=np.array(g_pts), g=g_slab, g_qep=g_slab_qep,
                        dos=dos_slab)

    # ---- bulk (n = 96, L = 40): two k-points, a few omegas -------------------
    wb = W.bulk_workload(n_k=16, n_omega=4096, n_layers=40)
    kb = np.array([37, 170])
    wb_sel = np.array([500, 1700, 2900])
    tb, pairs_b = [], []
    for ki in kb:
        lb = LeadBlocks(d00=wb.lead_l["d00"][ki], d01=wb.lead_l["d01"][ki], d10=wb.lead_l["d10"][ki])
        dv = Device1D(onsite_blocks=[wb.onsite[ki, 0]] * wb.n_layers,
                      coupling_blocks=[wb.coupling[ki, 0]] * (wb.n_layers - 1))
        for wi in wb_sel:
            tb.append(R.transmission(float(wb.omegas[wi]), dv, lb, lb, eta=wb.eta))
            pairs_b.append((wi, ki))
    lb = LeadBlocks(d00=wb.lead_l["d00"][kb[0]], d01=wb.lead_l["d01"][kb[0]], d10=wb.lead_l["d10"][kb[0]])
    gb = R.surface_gf(float(wb.omegas[1700]), lb.d00, lb.d01, lb.d10, eta=wb.eta)
    np.savez_compressed(OUT / "bulk.npz", omegas=wb.omegas[wb_sel], wsel=wb_sel, ksel=kb, pairs=np.array(pairs_b),
                        T=np.array(tb), d00=wb.lead_l["d00"][kb], d01=wb.lead_l["d01"][kb], n_layers=wb.n_layers,
                        eta=wb.eta, g=gb)

    # ---- negfpy test-suite systems ----------------------------------------
    cases = {}
    # matched chain plateau, L = 20 (tests/test_chain_transmission.py)
    wmax = 2.0
    om = np.linspace(0.2 * wmax, 0.8 * wmax, 9)
    d20 = device_perfect_chain(20, p)
    cases["chain_plateau_T"] = np.array([R.transmission(float(w), d20, lead, lead, eta=1e-8) for w in om])
    cases["chain_plateau_omega"] = om
    om = np.linspace(1.1 * wmax, 1.7 * wmax, 10)
    d16 = device_perfect_chain(16, p)
    cases["chain_outband_T"] = np.array([R.transmission(float(w), d16, lead, lead, eta=1e-8) for w in om])
    cases["chain_outband_omega"] = om
    # rectangular contact with a decoupled padding DOF (tests/test_interface_contacts.py)
    lead1 = LeadBlocks(d00=np.array([[2.0]], dtype=np.complex128), d01=np.array([[-1.0]], dtype=np.complex128))
    onsite = [np.diag([2.0, 100.0]).astype(np.complex128) for _ in range(4)]
    coupling = [np.diag([-1.0, 0.0]).astype(np.complex128) for _ in range(3)]
    cases["rect_T"] = np.array(R.transmission(1.0, Device1D(onsite, coupling), lead1, lead1, eta=1e-8,
                                              device_to_lead_left=np.array([[-1.0]]),
                                              device_to_lead_right=np.array([[-1.0]]),
                                              contact_left_indices=[0], contact_right_indices=[6]))
    # square lattice with k (tests/test_kspace_transport.py)
    sq = SquareLatticeParams(mass=1.0, spring_x=1.0, spring_y=0.5)
    sql, sqd = square_lattice_lead(sq), square_lattice_device(25, sq)
    kp = [(-np.pi,), (-np.pi / 3.0,), (0.0,), (np.pi / 3.0,), (np.pi,)]
    cases["square_kpoints"] = np.array(kp)
    cases["square_T"] = np.array([R.transmission(0.9, sqd, sql, sql, kpar=k) for k in kp])
    cases["square_kavg"] = np.array(R.transmission_kavg(0.9, sqd, sql, sql, kpoints=kp))
    # multi-DOF channel plateau (tests/test_multidof_transport.py)
    md = MultiDofCellParams(masses=np.ones(2), fc00=2.0 * np.eye(6), fc01=-np.eye(6), dof_per_atom=3)
    cases["multidof_T"] = np.array(R.transmission(1.0, multidof_device(30, md), multidof_lead_blocks(md),
                                                  multidof_lead_blocks(md), eta=1e-8))
    # omega_scale and a separate device eta on the slab system
    dv = Device1D(onsite_blocks=[wl.onsite[13, 0]] * 6, coupling_blocks=[wl.coupling[13, 0]] * 5)
    cases["slab_scaled_T"] = np.array(R.transmission(float(wl.omegas[900]), dv, lead_at[13], lead_at[13],
                                                     eta=wl.eta, eta_device=3.0 * wl.eta, omega_scale=1.7))
    # adaptive ladder on the chain (tests/test_chain_transmission.py)
    d14 = device_perfect_chain(14, p)
    tav, info = R.transmission_kavg_adaptive(1.0, d14, lead, lead, kpoints=[(), (), ()], eta_values=(1e-8, 1e-7),
                                             min_success_fraction=1.0)
    cases["chain_adaptive_T"] = np.array(tav)
    np.savez_compressed(OUT / "cases.npz", **cases)
    thermal(OUT)
    green(OUT)
    workflow(OUT)
    interface(OUT)
    dos(OUT)
    studies(OUT, studies_root)
    fcs(OUT, studies_root)
    dos_workflow(OUT, studies_root)
    print("wrote", sorted(p.name for p in OUT.glob("*.npz")))


if __name__ == "__main__":
    main()
