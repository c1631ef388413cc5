"""Parametric heterojunction device: spring constants -> k-space blocks.

A layered slab of ``ny x nz`` sites per principal layer (3 DOF each, block
order ``3 ny nz``), periodic in y (one transverse k), with free surfaces in
z.  Material A (layers ``< n_layers // 2``) occupies the sites with
z < ``nz_a``; the remaining sites of A layers are inert padding (no springs,
a stiff onsite pinning, so they carry no phonons in the frequency range, the
device trick of negfpy's ``tests/test_interface_contacts.py:36-37``).
Material B (the other layers) occupies every site.  Springs are central
NN/NNN springs as in ``workloads.spring_network``; A-A, B-B and A-B
(interface) bonds draw their constants from different ranges, masses per
material.  Both materials are periodic along x, so the leads are the
periodic crystals A (order 3 ny nz_a) and B (order 3 ny nz).

The device is described bond by bond.  A set of bonds around the interface
are parameters: ``theta`` (FP64) overrides their spring constants, and the
blocks are linear in theta:
    D(k; theta) = D_fixed(k) + sum_p theta_p dD(k)/dtheta_p.
``blocks(theta, kpoints, masses)`` evaluates them with torch, differentiable
in theta and in the device site masses (D = M^-1/2 Phi M^-1/2, the pinning
pin / m included), so gradients reach both through torch autograd from the
block gradients that the adjoint kernel provides.

The spring tables of the two materials are parameters too: ``phi_a`` and
``phi_b`` (one value per (site, neighbour vector) key, ``material_keys``)
set every A-A or B-B bond of the device (unless theta overrides it), the
half bonds at the device ends, and the periodic lead crystals, whose blocks
``lead_blocks_torch`` builds differentiably from them and from the masses of
device layer 0 (lead A) and layer L-1 (lead B).  Lead and device therefore
share parameters, and gradients reach them through the surface-GF adjoint.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from .workloads import _half_space_neighbours


@dataclass
class Contrib:
    """One 3x3 contribution of a bond to a block, per unit spring constant
    and before mass weighting: the block gets spring * raw / sqrt(m_a m_b)."""

    kind: np.ndarray    # 0 onsite block, 1 coupling block
    layer: np.ndarray   # block layer
    row: np.ndarray     # first DOF row
    col: np.ndarray     # first DOF column
    phase: np.ndarray   # transverse cell shift multiplying i ky
    raw: np.ndarray     # [m, 3, 3] real: +e e^T (self term) or -e e^T (pair term)
    ma: np.ndarray      # flat index (layer * n_sites + site) of the row site's mass
    mb: np.ndarray      # flat index of the column site's mass
    bond: np.ndarray    # bond index


class _deterministic:
    """Within the block builders, scatter-adds (index_add) in a fixed order on
    the GPU too, so that equal parameters give bitwise-equal blocks."""

    def __enter__(self):
        self.prev = torch.are_deterministic_algorithms_enabled()
        torch.use_deterministic_algorithms(True, warn_only=True)

    def __exit__(self, *exc):
        torch.use_deterministic_algorithms(self.prev)


class HeteroModel:
    def __init__(self, seed: int = 4, ny: int = 2, nz_a: int = 8, nz_b: int = 12, n_layers: int = 30,
                 n_params: int = 2000, pin: float = 100.0):
        rng = np.random.default_rng(seed)
        self.ny, self.nz, self.nz_a, self.L = ny, nz_b, nz_a, n_layers
        self.n_sites = ny * nz_b
        self.n = 3 * self.n_sites
        self.n_a = 3 * ny * nz_a
        self.split = n_layers // 2
        mass_a = rng.uniform(0.8, 1.2, size=(ny, nz_a))
        mass_b = rng.uniform(0.9, 1.4, size=(ny, nz_b))
        # Site tables: device site s = y * nz + z.
        self.site_y = np.repeat(np.arange(ny), nz_b)
        self.site_z = np.tile(np.arange(nz_b), ny)
        self.mass = np.ones((n_layers, self.n_sites))
        self.active = np.zeros((n_layers, self.n_sites), dtype=bool)
        for l in range(n_layers):
            for s in range(self.n_sites):
                y, z = self.site_y[s], self.site_z[s]
                if l < self.split:
                    if z < nz_a:
                        self.active[l, s] = True
                        self.mass[l, s] = mass_a[y, z]
                else:
                    self.active[l, s] = True
                    self.mass[l, s] = mass_b[y, z]
        self.pin = pin
        # Periodic spring tables per material, keyed by (site, neighbour vector).
        spr_a = {(s, d): rng.uniform(0.5, 1.5) for s in range(self.n_sites) for d in _half_space_neighbours()}
        spr_b = {(s, d): rng.uniform(0.8, 1.6) for s in range(self.n_sites) for d in _half_space_neighbours()}
        spr_i = {(s, d): rng.uniform(0.6, 1.4) for s in range(self.n_sites) for d in _half_space_neighbours()}
        self._spr = (spr_a, spr_b, spr_i)
        # Material spring tables as parameter vectors, one entry per (site, d).
        self.material_keys = [(s, d) for s in range(self.n_sites) for d in _half_space_neighbours()]
        self.key_index = {kd: i for i, kd in enumerate(self.material_keys)}
        self.phi0_a = np.array([spr_a[kd] for kd in self.material_keys])
        self.phi0_b = np.array([spr_b[kd] for kd in self.material_keys])
        # Bond instances of the device.  Layers -1 and n_layers stand for the
        # leads: a spring crossing the device boundary contributes only its
        # device-side self term (the rest is the lead coupling).
        la, a, lb, b, cy, ev, k0 = [], [], [], [], [], [], []
        src, key = [], []  # spring source of each bond: 0 fixed (interface), 1 phi_a, 2 phi_b
        for s in range(self.n_sites):  # lead A (layer -1) -> device layer 0
            if self.site_z[s] >= nz_a:
                continue
            for d in _half_space_neighbours():
                dx, dy, dz = d
                y2, z2 = self.site_y[s] + dy, self.site_z[s] + dz
                if dx != 1 or z2 < 0 or z2 >= nz_a:
                    continue
                c, y2 = divmod(y2, ny)
                s2 = y2 * nz_b + z2
                la.append(-1), a.append(s), lb.append(0), b.append(s2), cy.append(c)
                ev.append(np.asarray(d, float) / np.linalg.norm(d))
                k0.append(spr_a[(s, d)])
                src.append(1), key.append(self.key_index[(s, d)])
        for l in range(n_layers):
            for s in range(self.n_sites):
                if not self.active[l, s]:
                    continue
                for d in _half_space_neighbours():
                    dx, dy, dz = d
                    l2 = l + dx
                    y2, z2 = self.site_y[s] + dy, self.site_z[s] + dz
                    if z2 < 0 or z2 >= nz_b:
                        continue
                    c, y2 = divmod(y2, ny)
                    s2 = y2 * nz_b + z2
                    if l2 >= n_layers:  # device layer L-1 -> lead B (layer L)
                        la.append(l), a.append(s), lb.append(l2), b.append(s2), cy.append(c)
                        ev.append(np.asarray(d, float) / np.linalg.norm(d))
                        k0.append(spr_b[(s, d)])
                        src.append(2), key.append(self.key_index[(s, d)])
                        continue
                    if not self.active[l2, s2]:
                        continue
                    ma, mb = l < self.split, l2 < self.split
                    which = 1 if (ma and mb) else (2 if (not ma and not mb) else 0)
                    table = (spr_i, spr_a, spr_b)[which]
                    la.append(l), a.append(s), lb.append(l2), b.append(s2), cy.append(c)
                    ev.append(np.asarray(d, float) / np.linalg.norm(d))
                    k0.append(table[(s, d)])
                    src.append(which), key.append(self.key_index[(s, d)])
        self.bond_la, self.bond_a = np.array(la), np.array(a)
        self.bond_lb, self.bond_b = np.array(lb), np.array(b)
        self.bond_cy, self.bond_e, self.bond_k0 = np.array(cy), np.array(ev), np.array(k0)
        self.bond_src, self.bond_key = np.array(src), np.array(key)
        # Parameters: the bonds nearest to the interface layer boundary (never
        # the half bonds at the device ends).
        mid = self.split - 0.5
        dist = np.abs(0.5 * (self.bond_la + self.bond_lb) - mid)
        dist[(self.bond_la < 0) | (self.bond_lb >= n_layers)] = np.inf
        order = np.lexsort((np.arange(dist.size), dist))
        self.param_bonds = np.sort(order[:n_params])
        self.theta0 = self.bond_k0[self.param_bonds].copy()
        self.is_param = np.zeros(self.bond_k0.size, dtype=bool)
        self.is_param[self.param_bonds] = True
        self.contrib = self._contributions()
        self._lead_contrib = {m: self._lead_contributions(m) for m in ("A", "B")}

    # ---------------------------------------------------------------- blocks
    def _contributions(self) -> Contrib:
        kind, layer, row, col, phase, raw, ma, mb, bond = [], [], [], [], [], [], [], [], []
        ns = self.n_sites
        for i in range(self.bond_k0.size):
            la, a, lb, b = self.bond_la[i], self.bond_a[i], self.bond_lb[i], self.bond_b[i]
            e = self.bond_e[i]
            ee = np.outer(e, e)
            c = self.bond_cy[i]
            inside_a, inside_b = 0 <= la < self.L, 0 <= lb < self.L
            # self terms (device-side ends only)
            for (inside, l, s) in ((inside_a, la, a), (inside_b, lb, b)):
                if inside:
                    kind.append(0), layer.append(l), row.append(3 * s), col.append(3 * s), phase.append(0)
                    raw.append(ee), ma.append(l * ns + s), mb.append(l * ns + s), bond.append(i)
            if not (inside_a and inside_b):
                continue
            ia, ib = la * ns + a, lb * ns + b
            if la == lb:
                kind += [0, 0]
                layer += [la, la]
                row += [3 * a, 3 * b]
                col += [3 * b, 3 * a]
                phase += [c, -c]
                raw += [-ee, -ee]
                ma += [ia, ib]
                mb += [ib, ia]
                bond += [i, i]
            else:
                kind.append(1), layer.append(la), row.append(3 * a), col.append(3 * b), phase.append(c)
                raw.append(-ee), ma.append(ia), mb.append(ib), bond.append(i)
        return Contrib(np.array(kind), np.array(layer), np.array(row), np.array(col), np.array(phase, float),
                       np.array(raw), np.array(ma), np.array(mb), np.array(bond))

    def spring_values(self, theta: torch.Tensor, phi_a: torch.Tensor | None = None,
                      phi_b: torch.Tensor | None = None) -> torch.Tensor:
        """Spring constant of every device bond: the material tables phi_a /
        phi_b (default the model's) for A-A and B-B bonds and the half bonds
        at the ends, the fixed interface table otherwise, theta on the
        parameter bonds."""
        dev = theta.device
        kvals = torch.as_tensor(self.bond_k0, device=dev, dtype=torch.float64).clone()
        for which, phi in ((1, phi_a), (2, phi_b)):
            if phi is None:
                continue
            sel = np.flatnonzero(self.bond_src == which)
            kvals = kvals.index_put((torch.as_tensor(sel, device=dev),),
                                    phi.to(dev)[torch.as_tensor(self.bond_key[sel], device=dev)])
        return kvals.index_put((torch.as_tensor(self.param_bonds, device=dev),), theta.to(dev))

    def blocks(self, theta: torch.Tensor, kpoints, masses: torch.Tensor | None = None, device=None,
               phi_a: torch.Tensor | None = None, phi_b: torch.Tensor | None = None):
        """(onsite [K, L, n, n], coupling [K, L-1, n, n]) complex128 for spring
        values theta, material tables phi_a / phi_b and device site masses
        ``masses`` ``[L, ny*nz]`` (defaults the model's); differentiable in all
        of them with torch autograd.

        The spring contributions are summed with ``index_add`` in torch's
        deterministic mode, so equal parameters give bitwise-equal blocks."""
        with _deterministic():
            return self._blocks(theta, kpoints, masses, device, phi_a, phi_b)

    def _blocks(self, theta, kpoints, masses, device, phi_a, phi_b):
        dev = device or theta.device
        ky = torch.as_tensor(np.array([k[0] for k in kpoints], float), device=dev)
        K, L, n = ky.numel(), self.L, self.n
        m = torch.as_tensor(self.mass, device=dev, dtype=torch.float64) if masses is None else masses.to(dev)
        mflat = m.reshape(-1)
        kvals = self.spring_values(theta.to(dev), phi_a, phi_b)
        ct = self.contrib
        spring = kvals[torch.as_tensor(ct.bond, device=dev)]                      # [m]
        inv = torch.rsqrt(mflat[torch.as_tensor(ct.ma, device=dev)] * mflat[torch.as_tensor(ct.mb, device=dev)])
        ph = torch.exp(1j * ky[:, None] * torch.as_tensor(ct.phase, device=dev)[None, :])  # [K, m]
        val = ((spring * inv)[None, :, None, None] * ph[:, :, None, None]
               * torch.as_tensor(ct.raw, device=dev)[None])                         # [K, m, 3, 3]
        onsite = torch.zeros((K, L * n * n), dtype=torch.complex128, device=dev)
        coupling = torch.zeros((K, max(L - 1, 1) * n * n), dtype=torch.complex128, device=dev)
        ar = torch.arange(3, device=dev)
        r = torch.as_tensor(ct.row, device=dev)[:, None, None] + ar[None, :, None]
        c = torch.as_tensor(ct.col, device=dev)[:, None, None] + ar[None, None, :]
        lay = torch.as_tensor(ct.layer, device=dev)[:, None, None]
        flat = (lay * n * n + r * n + c).expand(-1, 3, 3)                          # [m, 3, 3]
        kind = torch.as_tensor(ct.kind, device=dev)
        for kd, tgt in ((0, onsite), (1, coupling)):
            sel = kind == kd
            if bool(sel.any()):
                idx = flat[sel].reshape(-1)
                tgt.index_add_(1, idx, val[:, sel].reshape(K, -1))
        # stiff pinning of the padding sites: pin / m on their 3 x 3 diagonal
        pl, ps = np.nonzero(~self.active)
        pin_val = self.pin / m[torch.as_tensor(pl, device=dev), torch.as_tensor(ps, device=dev)]   # [p]
        d = torch.arange(3, device=dev)
        idx = (torch.as_tensor(pl, device=dev)[:, None] * n * n
               + (3 * torch.as_tensor(ps, device=dev)[:, None] + d[None, :]) * (n + 1))          # [p, 3]
        pin_flat = torch.zeros(L * n * n, dtype=torch.float64, device=dev).index_add(
            0, idx.reshape(-1), pin_val[:, None].expand(-1, 3).reshape(-1))
        onsite = onsite.reshape(K, L, n, n) + pin_flat.reshape(L, n, n)[None]
        return onsite, coupling.reshape(K, max(L - 1, 1), n, n)

    # ------------------------------------------------------------ the leads
    def lead_blocks(self, material: str, kpoints) -> dict:
        """Periodic lead A or B: d00, d01, d10 [K, m, m] with A's sites in its own order."""
        spr_a, spr_b, _ = self._spr
        table = spr_a if material == "A" else spr_b
        nz = self.nz_a if material == "A" else self.nz
        sites = [(y, z) for y in range(self.ny) for z in range(nz)]
        index = {s: i for i, s in enumerate(sites)}
        m = 3 * len(sites)
        lay = 0 if material == "A" else self.L - 1
        mass = np.array([self.mass[lay, y * self.nz + z] for y, z in sites])
        K = len(kpoints)
        d00 = np.zeros((K, m, m), dtype=complex)
        d01 = np.zeros((K, m, m), dtype=complex)
        for ki, kp in enumerate(kpoints):
            ky = kp[0]
            for (y, z) in sites:
                s_dev = y * self.nz + z
                i = index[(y, z)]
                for d in _half_space_neighbours():
                    dx, dy, dz = d
                    y2, z2 = y + dy, z + dz
                    if z2 < 0 or z2 >= nz:
                        continue
                    c, y2 = divmod(y2, self.ny)
                    j = index[(y2, z2)]
                    e = np.asarray(d, float) / np.linalg.norm(d)
                    ee = table[(s_dev, d)] * np.outer(e, e)
                    d00[ki, 3 * i:3 * i + 3, 3 * i:3 * i + 3] += ee / mass[i]
                    d00[ki, 3 * j:3 * j + 3, 3 * j:3 * j + 3] += ee / mass[j]
                    w = -ee / np.sqrt(mass[i] * mass[j]) * np.exp(1j * ky * c)
                    if dx == 0:
                        d00[ki, 3 * i:3 * i + 3, 3 * j:3 * j + 3] += w
                        d00[ki, 3 * j:3 * j + 3, 3 * i:3 * i + 3] += np.conj(w)
                    else:
                        d01[ki, 3 * i:3 * i + 3, 3 * j:3 * j + 3] += w
        return {"d00": d00, "d01": d01, "d10": np.conj(np.swapaxes(d01, 1, 2)), "sites": sites}

    def _lead_contributions(self, material: str) -> dict:
        """Contribution table of the periodic lead's blocks, the same sums as
        ``lead_blocks``: per term its block (0 d00, 1 d01), 3x3 offset, phase
        shift, +-e e^T, the two masses (flat device index: layer 0 for A,
        layer L-1 for B) and the material key of its spring."""
        nz = self.nz_a if material == "A" else self.nz
        sites = [(y, z) for y in range(self.ny) for z in range(nz)]
        index = {st: i for i, st in enumerate(sites)}
        lay = 0 if material == "A" else self.L - 1
        t = {k: [] for k in ("blk", "row", "col", "phase", "raw", "ma", "mb", "key")}

        def add(blk, row, col, phase, raw, ma, mb, key):
            for k, v in zip(t, (blk, row, col, phase, raw, ma, mb, key)):
                t[k].append(v)

        for (y, z) in sites:
            s_dev = y * self.nz + z
            i = index[(y, z)]
            for d in _half_space_neighbours():
                dx, dy, dz = d
                y2, z2 = y + dy, z + dz
                if z2 < 0 or z2 >= nz:
                    continue
                c, y2 = divmod(y2, self.ny)
                j = index[(y2, z2)]
                e = np.asarray(d, float) / np.linalg.norm(d)
                ee = np.outer(e, e)
                key = self.key_index[(s_dev, d)]
                fi, fj = lay * self.n_sites + s_dev, lay * self.n_sites + y2 * self.nz + z2
                add(0, 3 * i, 3 * i, 0, ee, fi, fi, key)
                add(0, 3 * j, 3 * j, 0, ee, fj, fj, key)
                if dx == 0:
                    add(0, 3 * i, 3 * j, c, -ee, fi, fj, key)
                    add(0, 3 * j, 3 * i, -c, -ee, fj, fi, key)
                else:
                    add(1, 3 * i, 3 * j, c, -ee, fi, fj, key)
        out = {k: np.array(v) for k, v in t.items()}
        out["m"] = 3 * len(sites)
        return out

    def lead_blocks_torch(self, material: str, kpoints, phi: torch.Tensor | None = None,
                          masses: torch.Tensor | None = None, device=None) -> dict:
        """Lead A or B as torch tensors d00, d01, d10 = d01^H ``[K, m, m]``,
        differentiable in its material table ``phi`` (default the model's)
        and in the device masses (layer 0 for A, layer L-1 for B); equal to
        ``lead_blocks`` at the defaults.  Summed in torch's deterministic mode."""
        with _deterministic():
            return self._lead_blocks_torch(material, kpoints, phi, masses, device)

    def _lead_blocks_torch(self, material, kpoints, phi, masses, device):
        dev = device or (phi.device if phi is not None else (masses.device if masses is not None else "cpu"))
        ct = self._lead_contrib[material]
        if phi is None:
            phi = torch.as_tensor(self.phi0_a if material == "A" else self.phi0_b, device=dev)
        m = torch.as_tensor(self.mass, device=dev, dtype=torch.float64) if masses is None else masses.to(dev)
        mflat = m.reshape(-1)
        ky = torch.as_tensor(np.array([k[0] for k in kpoints], float), device=dev)
        K, mo = ky.numel(), ct["m"]
        t = lambda a: torch.as_tensor(a, device=dev)  # noqa: E731
        spring = phi.to(dev)[t(ct["key"])]
        inv = torch.rsqrt(mflat[t(ct["ma"])] * mflat[t(ct["mb"])])
        ph = torch.exp(1j * ky[:, None] * t(ct["phase"]).to(torch.float64)[None, :])
        val = (spring * inv)[None, :, None, None] * ph[:, :, None, None] * t(ct["raw"])[None]
        ar = torch.arange(3, device=dev)
        r = t(ct["row"])[:, None, None] + ar[None, :, None]
        c = t(ct["col"])[:, None, None] + ar[None, None, :]
        flat = (r * mo + c).expand(-1, 3, 3)
        out = []
        for b in (0, 1):
            sel = t(ct["blk"]) == b
            blk = torch.zeros((K, mo * mo), dtype=torch.complex128, device=dev)
            blk = blk.index_add(1, flat[sel].reshape(-1), val[:, sel].reshape(K, -1))
            out.append(blk.reshape(K, mo, mo))
        return {"d00": out[0], "d01": out[1], "d10": out[1].conj().transpose(-1, -2)}

    def omega_max(self, nk: int = 8) -> float:
        """Largest bulk phonon frequency of the two leads over a (kx, ky) sample."""
        ks = -np.pi + (np.arange(nk) + 0.5) * (2.0 * np.pi / nk)
        wmax = 0.0
        for mat in ("A", "B"):
            lb = self.lead_blocks(mat, [(k,) for k in ks])
            for kx in ks:
                d = lb["d00"] + lb["d01"] * np.exp(1j * kx) + lb["d10"] * np.exp(-1j * kx)
                d = 0.5 * (d + np.conj(np.swapaxes(d, 1, 2)))
                wmax = max(wmax, float(np.sqrt(max(np.linalg.eigvalsh(d).max(), 0.0))))
        return wmax

    def contact_left_indices(self) -> np.ndarray:
        """Device DOFs of layer 0 in lead A's DOF order."""
        idx = []
        for y in range(self.ny):
            for z in range(self.nz_a):
                s = y * self.nz + z
                idx += [3 * s, 3 * s + 1, 3 * s + 2]
        return np.array(idx)
