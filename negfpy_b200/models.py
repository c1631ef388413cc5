"""Block providers for the NEGF path: the 1D chain and the force-constant model.

``ChainParams``/``lead_blocks``/``device_perfect_chain``/``analytic_band_max``
restate negfpy ``models/chain.py:16-57``; ``MaterialKspaceParams`` with
``material_kspace_lead``/``material_kspace_device`` restate
``models/material_kspace.py:17-195`` (k-space blocks
``D(k) = M^-1/2 [sum_t Phi_t exp(i k.r_t)] M^-1/2``).

Besides the per-k callbacks negfpy uses, ``material_kspace_stack`` evaluates
the blocks for a whole k list at once as stacked arrays ``[K, n, n]``.  That
is the form the batched GPU path consumes: blocks are built once per k and
reused for every frequency, instead of once per (omega, k) point.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .types import Device1D, DeviceKSpace, KPar, LeadBlocks, LeadKSpace

Array = np.ndarray
Shift2D = tuple[int, int]


# ---------------------------------------------------------------- chain ----
@dataclass(frozen=True)
class ChainParams:
    mass: float
    spring: float


def lead_blocks(params: ChainParams) -> LeadBlocks:
    """1x1 lead blocks of a monatomic chain: d00 = 2k/m, d01 = -k/m."""
    return LeadBlocks(
        d00=np.array([[2.0 * params.spring / params.mass]], dtype=float),
        d01=np.array([[-params.spring / params.mass]], dtype=float),
    )


def device_perfect_chain(n_layers: int, params: ChainParams) -> Device1D:
    on = 2.0 * params.spring / params.mass
    cp = -params.spring / params.mass
    return Device1D(
        onsite_blocks=[np.array([[on]], dtype=float) for _ in range(n_layers)],
        coupling_blocks=[np.array([[cp]], dtype=float) for _ in range(n_layers - 1)],
    )


def device_mass_defect(n_layers: int, params: ChainParams, defect_index: int, defect_mass: float) -> Device1D:
    if defect_index < 0 or defect_index >= n_layers:
        raise ValueError("defect_index out of range")
    onsite = []
    for i in range(n_layers):
        m = defect_mass if i == defect_index else params.mass
        onsite.append(np.array([[2.0 * params.spring / m]], dtype=float))
    cp = -params.spring / params.mass
    return Device1D(onsite_blocks=onsite, coupling_blocks=[np.array([[cp]], dtype=float) for _ in range(n_layers - 1)])


def analytic_band_max(params: ChainParams) -> float:
    """Top of the chain's acoustic band, 2 sqrt(k/m)."""
    return float(2.0 * np.sqrt(params.spring / params.mass))


# ------------------------------------------------------ force constants ----
@dataclass(frozen=True)
class MaterialKspaceParams:
    """Force-constant terms for x transport with periodic y/z directions.

    ``fc00_terms``/``fc01_terms``/``fc10_terms`` map a transverse cell shift
    (dy, dz) to an (n_atoms*dof) square block; the k-space block is
    ``sum_(dy,dz) Phi(dy,dz) exp(i (ky dy + kz dz))``.  ``fc10_terms=None``
    means the Hermitian conjugate of the fc01 sum.
    """

    masses: Array
    fc00_terms: dict
    fc01_terms: dict
    fc10_terms: dict | None = None
    dof_per_atom: int = 3
    onsite_pinning: float = 0.0

    def __post_init__(self) -> None:
        masses = np.asarray(self.masses, dtype=float)
        if masses.ndim != 1 or masses.size == 0:
            raise ValueError("masses must be a non-empty 1D array.")
        if np.any(masses <= 0.0):
            raise ValueError("All masses must be positive.")
        if self.dof_per_atom <= 0:
            raise ValueError("dof_per_atom must be positive.")
        if len(self.fc00_terms) == 0:
            raise ValueError("fc00_terms must contain at least one term.")
        if len(self.fc01_terms) == 0:
            raise ValueError("fc01_terms must contain at least one term.")
        ndof = masses.size * self.dof_per_atom
        groups = [("fc00_terms", self.fc00_terms), ("fc01_terms", self.fc01_terms)]
        if self.fc10_terms is not None:
            if len(self.fc10_terms) == 0:
                raise ValueError("fc10_terms must be non-empty when provided.")
            groups.append(("fc10_terms", self.fc10_terms))
        for name, terms in groups:
            for key, block in terms.items():
                if len(key) != 2:
                    raise ValueError(f"{name} keys must be (dy, dz).")
                if np.shape(block) != (ndof, ndof):
                    raise ValueError(f"{name} blocks must have shape (n_atoms*dof, n_atoms*dof).")

    @property
    def n_atoms(self) -> int:
        return int(np.asarray(self.masses).size)

    @property
    def ndof(self) -> int:
        return self.n_atoms * self.dof_per_atom


def parse_ky_kz(kpar: KPar) -> tuple[float, float]:
    if kpar is None or len(kpar) == 0:
        return 0.0, 0.0
    if len(kpar) > 2:
        raise ValueError("kpar must contain at most two transverse components: (ky,) or (ky, kz).")
    if len(kpar) == 1:
        return float(kpar[0]), 0.0
    return float(kpar[0]), float(kpar[1])


def _phase_sum_stack(terms: dict, ky: Array, kz: Array) -> Array:
    """sum_t Phi_t exp(i(ky dy + kz dz)) for every k at once -> [K, n, n]."""
    keys = list(terms.keys())
    blocks = np.stack([np.asarray(terms[k], dtype=np.complex128) for k in keys])  # [T, n, n]
    shifts = np.asarray(keys, dtype=float)  # [T, 2]
    phase = np.exp(1j * (np.outer(ky, shifts[:, 0]) + np.outer(kz, shifts[:, 1])))  # [K, T]
    return np.einsum("kt,tij->kij", phase, blocks)


def _inv_sqrt_mass(masses: Array, dof: int) -> Array:
    return 1.0 / np.sqrt(np.repeat(np.asarray(masses, dtype=float), dof))


def material_kspace_stack(params: MaterialKspaceParams, kpoints: list, layer_masses: Array | None = None,
                          n_layers: int | None = None) -> dict:
    """Lead and device blocks of a force-constant model for a list of k.

    Returns ``{"d00","d01","d10"}: [K, n, n]`` for the lead, and when
    ``n_layers`` is given also ``"onsite": [K, L, n, n]`` and
    ``"coupling": [K, L-1, n, n]`` for the device (per-layer masses from
    ``layer_masses`` of shape ``(L, n_atoms)``).  The arithmetic is the same
    as the per-k builders of negfpy ``models/material_kspace.py:99-193``.
    """
    kk = [parse_ky_kz(k) for k in kpoints]
    ky = np.array([a for a, _ in kk], dtype=float)
    kz = np.array([b for _, b in kk], dtype=float)
    phi00 = _phase_sum_stack(params.fc00_terms, ky, kz)
    if params.onsite_pinning != 0.0:
        phi00 = phi00 + params.onsite_pinning * np.eye(params.ndof, dtype=np.complex128)[None]
    phi01 = _phase_sum_stack(params.fc01_terms, ky, kz)
    if params.fc10_terms is None:
        phi10 = np.conj(np.swapaxes(phi01, 1, 2))
    else:
        phi10 = _phase_sum_stack(params.fc10_terms, ky, kz)
    m = _inv_sqrt_mass(params.masses, params.dof_per_atom)
    out = {
        "d00": m[None, :, None] * phi00 * m[None, None, :],
        "d01": m[None, :, None] * phi01 * m[None, None, :],
        "d10": m[None, :, None] * phi10 * m[None, None, :],
    }
    if n_layers is not None:
        if layer_masses is None:
            lm = np.repeat(np.asarray(params.masses, dtype=float)[None, :], n_layers, axis=0)
        else:
            lm = np.asarray(layer_masses, dtype=float)
        ms = np.stack([_inv_sqrt_mass(lm[i], params.dof_per_atom) for i in range(n_layers)])  # [L, n]
        out["onsite"] = ms[None, :, :, None] * phi00[:, None] * ms[None, :, None, :]
        out["coupling"] = ms[None, :-1, :, None] * phi01[:, None] * ms[None, 1:, None, :]
    return out


def _blocks_at(params: MaterialKspaceParams, kpar: KPar, ml: Array, mr: Array):
    st = material_kspace_stack(params, [kpar if kpar is not None else ()])
    # Re-weight with the requested masses (the stack used params.masses).
    m0 = _inv_sqrt_mass(params.masses, params.dof_per_atom)
    a = _inv_sqrt_mass(ml, params.dof_per_atom) / m0
    b = _inv_sqrt_mass(mr, params.dof_per_atom) / m0
    d00 = a[:, None] * st["d00"][0] * a[None, :]
    d01 = a[:, None] * st["d01"][0] * b[None, :]
    d10 = b[:, None] * st["d10"][0] * a[None, :]
    return d00, d01, d10


def material_kspace_lead(params: MaterialKspaceParams) -> LeadKSpace:
    """k-dependent lead blocks (d00, d01, d10) of a force-constant model."""

    def _builder(kpar: KPar):
        return _blocks_at(params, kpar, params.masses, params.masses)

    _builder.kspace_params = params  # lets the batched path build every k on the GPU
    return LeadKSpace(blocks_builder=_builder)


def material_kspace_device(n_layers: int, params: MaterialKspaceParams, layer_masses: Array | None = None) -> DeviceKSpace:
    """k-dependent device of ``n_layers`` principal layers with optional per-layer masses."""
    if n_layers <= 0:
        raise ValueError("n_layers must be positive.")
    if layer_masses is None:
        masses = np.repeat(np.asarray(params.masses, dtype=float)[None, :], n_layers, axis=0)
    else:
        masses = np.asarray(layer_masses, dtype=float)
        if masses.shape != (n_layers, params.n_atoms):
            raise ValueError("layer_masses shape must be (n_layers, n_atoms).")
        if np.any(masses <= 0.0):
            raise ValueError("All layer_masses entries must be positive.")

    def _builder(kpar: KPar) -> Device1D:
        st = material_kspace_stack(params, [kpar if kpar is not None else ()], layer_masses=masses, n_layers=n_layers)
        return Device1D(onsite_blocks=list(st["onsite"][0]), coupling_blocks=list(st["coupling"][0]))

    _builder.kspace_params = params
    _builder.kspace_device = {"n_layers": int(n_layers), "layer_masses": None if layer_masses is None else masses}
    return DeviceKSpace(device_builder=_builder)


def interface_terms(params: MaterialKspaceParams) -> tuple[dict, dict]:
    """Force-constant terms of the two lead couplings of the IFC transport
    set-up (negfpy ``workflows/ifc_bulk.py:690-711``): ``(left, right)``.

    With FC10 the given fc10 terms, or {(-dy, -dz): FC01(dy, dz)^H} when
    there are none, the left lead's d01 sums FC10(dy, dz) and the right
    lead's sums FC10(dy, dz)^T at the shift (-dy, -dz).
    """
    if params.fc10_terms is None:
        fc10 = {(-dy, -dz): np.asarray(v, dtype=np.complex128).conj().T for (dy, dz), v in params.fc01_terms.items()}
    else:
        fc10 = {key: np.asarray(v, dtype=np.complex128) for key, v in params.fc10_terms.items()}
    right = {(-dy, -dz): v.T for (dy, dz), v in fc10.items()}
    return dict(fc10), right


def interface_contacts(params: MaterialKspaceParams):
    """Leads and device couplings of the IFC transport set-up, as negfpy's
    ``_build_interface_contacts`` (``workflows/ifc_bulk.py:690-742``).

    Returns ``(lead_left, lead_right, device_to_lead_left, device_to_lead_right)``:
    two ``LeadKSpace`` with blocks (d00, d01, d01^H), where d00 = M (Phi00(k)
    + pinning) M and d01 = M K01(k) M over the terms of ``interface_terms``
    (M = diag(m^-1/2)), and the couplings V_R(k) = d01 of the right lead and
    V_L(k) = V_R(k)^H.  Each builder is tagged so that the batched path can
    build every k of the same set-up on the GPU.
    """
    left_terms, right_terms = interface_terms(params)
    m = _inv_sqrt_mass(params.masses, params.dof_per_atom)
    pin = float(params.onsite_pinning)

    def _weighted(terms: dict, kpar: KPar, pinning: float = 0.0) -> Array:
        ky, kz = parse_ky_kz(kpar)
        phi = _phase_sum_stack(terms, np.array([ky]), np.array([kz]))[0]
        if pinning != 0.0:
            phi = phi + pinning * np.eye(params.ndof, dtype=np.complex128)
        return m[:, None] * phi * m[None, :]

    def _lead(terms: dict):
        def _builder(kpar: KPar):
            d00 = _weighted(params.fc00_terms, kpar, pin)
            d01 = _weighted(terms, kpar)
            return d00, d01, d01.conj().T
        return _builder

    def _vdl_right(kpar: KPar) -> Array:
        return _weighted(right_terms, kpar)

    def _vdl_left(kpar: KPar) -> Array:
        return _vdl_right(kpar).conj().T

    token = object()  # ties the four pieces of one set-up together
    left, right = _lead(left_terms), _lead(right_terms)
    for fn, role in ((left, "left"), (right, "right"), (_vdl_left, "vdl_left"), (_vdl_right, "vdl_right")):
        fn.kspace_interface = (token, params, role)
    return LeadKSpace(blocks_builder=left), LeadKSpace(blocks_builder=right), _vdl_left, _vdl_right
