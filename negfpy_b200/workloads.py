"""Seeded synthetic workloads for the batched NEGF path.

The spring network is new code (negfpy has no random-structure generator):
atoms sit on a simple-cubic grid; every nearest-neighbour (|d| = 1) and
next-nearest-neighbour (|d| = sqrt 2) pair is joined by a central spring of
constant k ~ U[lo, hi]; masses are m ~ U[lo, hi].  A central spring between
atoms a, b with unit bond vector e adds ``k e e^T`` to both self blocks and
``-k e e^T`` to the a-b and b-a blocks, so the force constants obey the
acoustic sum rule and the dynamical matrix is positive semidefinite by
construction (the energy is a sum of squares).  The result is emitted as
``MaterialKspaceParams`` fc00/fc01 terms keyed by the transverse cell shift
(dy, dz), the form negfpy's ``models/material_kspace.py`` consumes.

The principal layer is one lattice spacing thick along x (transport), so
NN and NNN springs only reach the adjacent layer.  Transversally the layer
holds ``ny x nz`` sites; a direction is either periodic (a k component) or
finite with free surfaces.

Frequency grids follow negfpy's conventions: shifted k lines
``k_j = -pi + (j + 1/2) 2 pi / nk`` (``workflows/ifc_bulk.py:154-173``) and
omega_max estimated as the largest sqrt(eig D(kx, k_par)) over a k sample
(``workflows/ifc_bulk.py:229-257``).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from itertools import product

import numpy as np

from .models import MaterialKspaceParams, material_kspace_stack

# Physical constants (SI) used for kappa, as in negfpy ``workflows/ifc_bulk.py:53-56``.
HBAR_J_S = 1.054_571_817e-34
KB_J_K = 1.380_649e-23


def _half_space_neighbours() -> list[tuple[int, int, int]]:
    """One representative of each +-pair of NN and NNN displacement vectors."""
    vecs = []
    for d in product((-1, 0, 1), repeat=3):
        s = abs(d[0]) + abs(d[1]) + abs(d[2])
        if s == 0 or s == 3:
            continue
        if d > (0, 0, 0):  # lexicographic half space
            vecs.append(d)
    return vecs


def spring_network(
    seed: int,
    ny: int,
    nz: int,
    periodic_y: bool = True,
    periodic_z: bool = False,
    spring_range: tuple[float, float] = (0.5, 1.5),
    mass_range: tuple[float, float] = (0.8, 1.2),
) -> MaterialKspaceParams:
    """Random NN+NNN central-spring network with ``ny*nz`` atoms per layer (3 DOF each)."""
    rng = np.random.default_rng(seed)
    n_atoms = ny * nz
    ndof = 3 * n_atoms
    masses = rng.uniform(mass_range[0], mass_range[1], size=n_atoms)

    def atom(y: int, z: int) -> int:
        return y * nz + z

    fc00: dict[tuple[int, int], np.ndarray] = {}
    fc01: dict[tuple[int, int], np.ndarray] = {}

    def add(terms, key, a, b, blk):
        if key not in terms:
            terms[key] = np.zeros((ndof, ndof), dtype=float)
        terms[key][3 * a:3 * a + 3, 3 * b:3 * b + 3] += blk

    for y, z in product(range(ny), range(nz)):
        a = atom(y, z)
        for d in _half_space_neighbours():
            dx, dy, dz = d
            yy, zz = y + dy, z + dz
            if periodic_y:
                cy, yy = divmod(yy, ny)
            else:
                if yy < 0 or yy >= ny:
                    continue
                cy = 0
            if periodic_z:
                cz, zz = divmod(zz, nz)
            else:
                if zz < 0 or zz >= nz:
                    continue
                cz = 0
            b = atom(yy, zz)
            k = rng.uniform(spring_range[0], spring_range[1])
            e = np.asarray(d, dtype=float) / np.linalg.norm(d)
            ee = k * np.outer(e, e)
            # self terms (acoustic sum rule)
            add(fc00, (0, 0), a, a, ee)
            add(fc00, (0, 0), b, b, ee)
            # a (layer 0, cell 0) <-> b (layer dx, cell (cy, cz))
            if dx == 0:
                add(fc00, (cy, cz), a, b, -ee)
                add(fc00, (-cy, -cz), b, a, -ee)
            else:  # dx == +1 by the half-space choice when dx != 0
                add(fc01, (cy, cz), a, b, -ee)
    # A layer with dx=+1 bonds only towards +x is enough: fc10 = fc01^H.
    return MaterialKspaceParams(masses=masses, fc00_terms=fc00, fc01_terms=fc01, dof_per_atom=3)


def kline(nk: int) -> np.ndarray:
    """Shifted 1D k mesh (even nk) or Gamma for nk == 1."""
    if nk == 1:
        return np.zeros(1)
    return -np.pi + (np.arange(nk, dtype=float) + 0.5) * (2.0 * np.pi / nk)


def kgrid(nky: int, nkz: int = 0) -> list[tuple[float, ...]]:
    if nkz == 0:
        return [(float(v),) for v in kline(nky)]
    return [(float(a), float(b)) for a in kline(nky) for b in kline(nkz)]


def estimate_omega_max(params: MaterialKspaceParams, nk: int = 8, two_d: bool = False) -> float:
    """Largest phonon frequency over a (kx, k_par) sample of the bulk lead."""
    kxs = kline(nk)
    kps = kgrid(nk, nk) if two_d else kgrid(nk)
    st = material_kspace_stack(params, kps)
    wmax = 0.0
    for kx in kxs:
        d = st["d00"] + st["d01"] * np.exp(1j * kx) + st["d10"] * np.exp(-1j * kx)
        d = 0.5 * (d + np.conj(np.swapaxes(d, 1, 2)))
        ev = np.linalg.eigvalsh(d)
        wmax = max(wmax, float(np.sqrt(max(ev.max(), 0.0))))
    return wmax


@dataclass
class Workload:
    """Stacked blocks and grids of one (omega, k) batch workload.

    ``lead_l``/``lead_r``: dicts of ``d00/d01/d10`` arrays ``[K, n, n]``;
    ``onsite``: ``[K, L, n, n]`` (or ``[K, 1, n, n]`` with ``uniform_layers``);
    ``coupling``: ``[K, L-1, n, n]`` (or ``[K, 1, n, n]``); ``omegas``: ``[W]``;
    ``kpoints``: K tuples; ``eta`` / ``eta_device``: scalars.
    """

    name: str
    omegas: np.ndarray
    kpoints: list
    lead_l: dict
    lead_r: dict
    onsite: np.ndarray
    coupling: np.ndarray
    n_layers: int
    eta: float
    eta_device: float | None = None
    omega_max: float = 1.0
    omega_unit_rad_s: float = 1.0
    same_leads: bool = True
    uniform_layers: bool = False
    vl: np.ndarray | None = None  # [K, n_dev, n_lead_l] or None (default coupling)
    vr: np.ndarray | None = None
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.onsite.shape[-1])

    @property
    def n_points(self) -> int:
        return len(self.omegas) * len(self.kpoints)


def omega_unit_for(omega_max: float, thz: float = 15.0) -> float:
    """rad/s per model frequency unit so that omega_max maps to 2 pi * thz THz."""
    return 2.0 * np.pi * thz * 1e12 / omega_max


def chain_workload(n_omega: int = 1000, n_layers: int = 8) -> Workload:
    """1D monatomic chain, m = k = 1, midpoint omega grid on (0, 2), eta = 1e-8."""
    om = (np.arange(n_omega, dtype=float) + 0.5) * (2.0 / n_omega)
    d00 = np.full((1, 1, 1), 2.0, dtype=np.complex128)
    d01 = np.full((1, 1, 1), -1.0, dtype=np.complex128)
    lead = {"d00": d00, "d01": d01, "d10": d01.copy()}
    onsite = np.full((1, n_layers, 1, 1), 2.0, dtype=np.complex128)
    coupling = np.full((1, max(n_layers - 1, 1), 1, 1), -1.0, dtype=np.complex128)
    return Workload("chain_n1_L%d_W%d" % (n_layers, n_omega), om, [()], lead, lead, onsite, coupling,
                    n_layers, eta=1e-8, omega_max=2.0, omega_unit_rad_s=omega_unit_for(2.0))


def slab_workload(seed: int = 2, n_k: int = 64, n_omega: int = 2048, n_layers: int = 20,
                  ny: int = 2, nz: int = 8, uniform_layers: bool = True) -> Workload:
    """Quasi-2D slab: 16 atoms x 3 DOF (n = 48), 1D k line, identical device layers."""
    params = spring_network(seed, ny=ny, nz=nz, periodic_y=True, periodic_z=False)
    kps = kgrid(n_k)
    wmax = estimate_omega_max(params, nk=8, two_d=False)
    st = material_kspace_stack(params, kps, n_layers=1)
    lead = {"d00": st["d00"], "d01": st["d01"], "d10": st["d10"]}
    onsite = st["onsite"]  # [K, 1, n, n]; identical layers
    coupling = st["d01"][:, None]
    if not uniform_layers:
        onsite = np.repeat(onsite, n_layers, axis=1)
        coupling = np.repeat(coupling, n_layers - 1, axis=1)
    om = (np.arange(n_omega, dtype=float) + 1.0) * (1.05 * wmax / n_omega)
    return Workload("slab_n%d_L%d_K%d_W%d" % (3 * ny * nz, n_layers, n_k, n_omega), om, kps, lead, lead,
                    onsite, coupling, n_layers, eta=1e-6 * wmax * wmax, omega_max=wmax,
                    omega_unit_rad_s=omega_unit_for(wmax), uniform_layers=uniform_layers,
                    meta={"seed": seed, "ny": ny, "nz": nz})


def bulk_workload(seed: int = 3, n_k: int = 16, n_omega: int = 4096, n_layers: int = 40,
                  ny: int = 4, nz: int = 8, uniform_layers: bool = True) -> Workload:
    """3D bulk-like: 32 atoms x 3 DOF (n = 96), 2D k grid, identical device layers."""
    params = spring_network(seed, ny=ny, nz=nz, periodic_y=True, periodic_z=True)
    kps = kgrid(n_k, n_k)
    wmax = estimate_omega_max(params, nk=6, two_d=True)
    st = material_kspace_stack(params, kps, n_layers=1)
    lead = {"d00": st["d00"], "d01": st["d01"], "d10": st["d10"]}
    onsite = st["onsite"]
    coupling = st["d01"][:, None]
    if not uniform_layers:
        onsite = np.repeat(onsite, n_layers, axis=1)
        coupling = np.repeat(coupling, n_layers - 1, axis=1)
    om = (np.arange(n_omega, dtype=float) + 1.0) * (1.05 * wmax / n_omega)
    return Workload("bulk_n%d_L%d_K%d_W%d" % (3 * ny * nz, n_layers, n_k * n_k, n_omega), om, kps, lead, lead,
                    onsite, coupling, n_layers, eta=1e-6 * wmax * wmax, omega_max=wmax,
                    omega_unit_rad_s=omega_unit_for(wmax), uniform_layers=uniform_layers,
                    meta={"seed": seed, "ny": ny, "nz": nz})


def subsample(wl: Workload, omega_idx, k_idx) -> Workload:
    """A smaller workload on a subset of the omega grid and k list (same blocks)."""
    oi = np.asarray(omega_idx, dtype=int)
    ki = np.asarray(k_idx, dtype=int)
    sel = lambda d: {key: v[ki] for key, v in d.items()}  # noqa: E731
    return Workload(wl.name + "_sub", wl.omegas[oi], [wl.kpoints[i] for i in ki], sel(wl.lead_l), sel(wl.lead_r),
                    wl.onsite[ki], wl.coupling[ki], wl.n_layers, wl.eta, wl.eta_device, wl.omega_max,
                    wl.omega_unit_rad_s, wl.same_leads, wl.uniform_layers,
                    None if wl.vl is None else wl.vl[ki], None if wl.vr is None else wl.vr[ki], dict(wl.meta))


# Block orders of the uneven batch and the (ny, nz) atom grid of each (3 DOF per atom).
UNEVEN_SHAPES = {24: (2, 4), 48: (4, 4), 72: (4, 6), 96: (4, 8), 120: (4, 10), 192: (8, 8)}


def uneven_workload(seed: int = 5, n_systems: int = 64, n_omega: int = 1024, k_range: tuple[int, int] = (1, 256),
                    layer_range: tuple[int, int] = (10, 60), orders=tuple(UNEVEN_SHAPES)) -> list[Workload]:
    """Independent systems for one uneven batch: block orders drawn uniformly
    from ``orders``, lengths uniformly from ``layer_range`` layers and 1D k
    lines of ``k_range`` points, each a seeded NN+NNN spring network (slab,
    periodic in y) with its own omega grid of ``n_omega`` points up to
    1.05 omega_max and eta = 1e-6 omega_max^2.  Leads are the device material
    (identical layers)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_systems):
        n = int(rng.choice(orders))
        L = int(rng.integers(layer_range[0], layer_range[1] + 1))
        K = int(rng.integers(k_range[0], k_range[1] + 1))
        ny, nz = UNEVEN_SHAPES[n]
        params = spring_network(seed * 1000 + i, ny=ny, nz=nz, periodic_y=True, periodic_z=False)
        kps = kgrid(K)
        wmax = estimate_omega_max(params, nk=4, two_d=False)
        st = material_kspace_stack(params, kps, n_layers=1)
        lead = {"d00": st["d00"], "d01": st["d01"], "d10": st["d10"]}
        om = (np.arange(n_omega, dtype=float) + 1.0) * (1.05 * wmax / n_omega)
        out.append(Workload("uneven%d_n%d_L%d_K%d_W%d" % (i, n, L, K, n_omega), om, kps, lead, lead, st["onsite"],
                            st["d01"][:, None], L, eta=1e-6 * wmax * wmax, omega_max=wmax,
                            omega_unit_rad_s=omega_unit_for(wmax), uniform_layers=True,
                            meta={"seed": seed * 1000 + i, "ny": ny, "nz": nz}))
    return out
