"""Seeded synthetic systems with the shapes, sizes and value distributions of the
benchmark configurations (no structure files are available, so these stand in for them).

Each generator returns (topology, positions) where `topology` has the layout of RainMD's
`parsePrmtop` result (shared/amber/prmtop.js:363-395), ready for `build_system`.

  water_box(n)             ⌊n/3⌋ rigid TIP3P waters plus Na+ (and Cl-) for the remainder,
                           cubic, at 0.997 g/cm^3, jittered lattice, random orientations
  solvated_chain(n, m)     an m-atom flexible chain solute (charges N(0, 0.3) shifted to a
                           net -1, one Na+ counter-ion), bonds 1.0-1.5 Å with
                           k = 300 kcal/mol/Å^2 (AMBER k(r-r0)^2), angles 109.5° with k = 50,
                           one three-term torsion per dihedral, in TIP3P water
  batch(count, ...)        uneven solvated systems, sizes log-uniform between two bounds

TIP3P: O -0.834 e, H +0.417 e, O-H 0.9572 Å, H-O-H 104.52° (H-H 1.5136 Å),
sigma_O 3.15061 Å, epsilon_O 0.1521 kcal/mol, no LJ on H. Chain atoms are carbon-like
(12.011 amu, sigma 3.4 Å, epsilon 0.086 kcal/mol); Na+ and Cl- use sigma 2.439/4.478 Å,
epsilon 0.0874393/0.0355910 kcal/mol. Unlike-pair LJ uses the Lorentz-Berthelot rule.
"""
from __future__ import annotations

import math

import numpy as np

from .amber import ANGLE_K_SCALE, BOND_K_SCALE, ENERGY_SCALE

AMU_PER_NM3_TO_G_PER_CM3 = 1.66053906660e-3
O_H = 0.09572
H_H = 0.15136
WATER_MASS = (15.9994, 1.008, 1.008)

# type: (mass, charge, sigma nm, epsilon kJ/mol, atomic number, residue)
TYPES = {
    "OW": (15.9994, -0.834, 0.315061, 0.1521 * ENERGY_SCALE, 8),
    "HW": (1.008, 0.417, 0.1, 0.0, 1),
    "C": (12.011, 0.0, 0.34, 0.086 * ENERGY_SCALE, 6),
    "NA": (22.98977, 1.0, 0.2439, 0.0874393 * ENERGY_SCALE, 11),
    "CL": (35.453, -1.0, 0.4478, 0.0355910 * ENERGY_SCALE, 17),
}
TYPE_ORDER = ["OW", "HW", "C", "NA", "CL"]


def _lj_tables():
    n = len(TYPE_ORDER)
    a = np.zeros(n * n)
    b = np.zeros(n * n)
    for i, ti in enumerate(TYPE_ORDER):
        for j, tj in enumerate(TYPE_ORDER):
            si, ei = TYPES[ti][2], TYPES[ti][3]
            sj, ej = TYPES[tj][2], TYPES[tj][3]
            eps = math.sqrt(ei * ej)
            sig = 0.5 * (si + sj)
            a[n * i + j] = 4 * eps * sig ** 12
            b[n * i + j] = 4 * eps * sig ** 6
    return a, b


def _random_rotations(rng, count):
    q = rng.normal(size=(count, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], 1)


def _water_template():
    half = math.radians(104.52) / 2
    # O at the origin, H in the xy plane
    return np.array([[0.0, 0.0, 0.0],
                     [O_H * math.sin(half), O_H * math.cos(half), 0.0],
                     [-O_H * math.sin(half), O_H * math.cos(half), 0.0]])


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def _unit(v):
    n = math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
    return (v[0] / n, v[1] / n, v[2] / n), n


def _chain(rng, count, box=None):
    """A self-avoiding random walk with bond lengths 1.0-1.5 Å and 109.5° angles: every atom
    at least 3 Å from all but its two predecessors, by minimum image when `box` is given (a
    long chain in a small periodic box must not meet its own images). Random dihedrals are
    tried 16 at a time, up to 192 per step: the first that clears is taken, else the one that
    comes closest."""
    pos = np.zeros((count, 3))
    lengths = rng.uniform(0.10, 0.15, size=max(count - 1, 1))
    theta = math.radians(109.5)
    c_t, s_t = math.cos(math.pi - theta), math.sin(math.pi - theta)
    direction = np.array([1.0, 0.0, 0.0])
    previous = np.array([0.0, 1.0, 0.0])
    for k in range(1, count):
        axis = np.cross(direction, previous)
        norm = np.linalg.norm(axis)
        if norm < 1e-8:
            axis = np.cross(direction, rng.normal(size=3))
            norm = np.linalg.norm(axis)
        axis /= norm
        perp = np.cross(axis, direction)
        best, best_d2 = None, -1.0
        for _ in range(12):
            phi = rng.uniform(-math.pi, math.pi, size=16)
            # new directions at angle (pi - theta) from the current one, azimuths phi
            new = c_t * direction + s_t * (np.cos(phi)[:, None] * axis + np.sin(phi)[:, None] * perp)
            new /= np.linalg.norm(new, axis=1)[:, None]
            cand = pos[k - 1] + lengths[k - 1] * new
            if k < 3:
                best = (new[0], cand[0])
                break
            d = pos[None, :k - 2, :] - cand[:, None, :]
            if box is not None:
                d -= box * np.round(d / box)
            d2 = np.min(np.einsum("cka,cka->ck", d, d), axis=1)
            clear = np.nonzero(d2 > 0.09)[0]
            pick = int(clear[0]) if len(clear) else int(np.argmax(d2))
            if d2[pick] > best_d2:
                best, best_d2 = (new[pick], cand[pick]), float(d2[pick])
            if len(clear):
                break
        new_dir, candidate = best
        previous, direction = direction, new_dir
        pos[k] = candidate
    return pos - pos.mean(axis=0), lengths


class _Builder:
    def __init__(self):
        self.types, self.charges, self.masses, self.z, self.res, self.resnames = [], [], [], [], [], []
        self.pos = []
        self.bonds, self.angles, self.dihedrals = [], [], []
        self.excl: dict = {}
        self.mol = []
        self.nmol = 0

    def atom(self, kind, position, charge=None, residue=0):
        mass, q, _, _, z = TYPES[kind]
        self.types.append(TYPE_ORDER.index(kind))
        self.charges.append(q if charge is None else charge)
        self.masses.append(mass)
        self.z.append(z)
        self.res.append(residue)
        self.pos.append(position)
        self.mol.append(self.nmol)
        return len(self.types) - 1

    def exclude(self, a, b):
        lo, hi = min(a, b), max(a, b)
        self.excl.setdefault(lo, set()).add(hi)

    def add_water(self, origin, rotation):
        r = len(self.resnames)
        self.resnames.append("WAT")
        t = _water_template() @ rotation.T + origin
        o = self.atom("OW", t[0], residue=r)
        h1 = self.atom("HW", t[1], residue=r)
        h2 = self.atom("HW", t[2], residue=r)
        k = 553.0  # kcal/mol/Å^2, AMBER TIP3P
        self.bonds += [(o, h1, k, O_H), (o, h2, k, O_H), (h1, h2, k, H_H)]
        self.exclude(o, h1)
        self.exclude(o, h2)
        self.exclude(h1, h2)
        self.nmol += 1

    def add_ion(self, kind, origin):
        r = len(self.resnames)
        self.resnames.append("Na+" if kind == "NA" else "Cl-")
        self.atom(kind, origin, residue=r)
        self.nmol += 1

    def add_chain(self, rng, positions, lengths, net_charge=-1.0):
        r = len(self.resnames)
        self.resnames.append("CHN")
        count = len(positions)
        q = rng.normal(0.0, 0.3, size=count)
        q += (net_charge - q.sum()) / count
        first = len(self.types)
        for k in range(count):
            self.atom("C", positions[k], charge=float(q[k]), residue=r)
        idx = list(range(first, first + count))
        for k in range(count - 1):
            self.bonds.append((idx[k], idx[k + 1], 300.0, float(lengths[k])))
        for k in range(count - 2):
            self.angles.append((idx[k], idx[k + 1], idx[k + 2], 50.0, math.radians(109.5)))
        for k in range(count - 3):
            for n, barrier, phase in ((1, 0.20, 0.0), (2, 0.25, math.pi), (3, 0.18, 0.0)):
                self.dihedrals.append((idx[k], idx[k + 1], idx[k + 2], idx[k + 3], barrier, n, phase,
                                       n == 1))
        for k in range(count):
            for d in (1, 2, 3):
                if k + d < count:
                    self.exclude(idx[k], idx[k + d])
        self.nmol += 1

    def topology(self, box_length):
        n = len(self.types)
        lj_a, lj_b = _lj_tables()
        excl_start = np.zeros(n + 1, dtype=np.int32)
        partners = []
        for atom in range(n):
            excl_start[atom] = len(partners)
            partners.extend(sorted(self.excl.get(atom, ())))
        excl_start[n] = len(partners)
        bonds = np.array(self.bonds, dtype=np.float64).reshape(-1, 4)
        angles = np.array(self.angles, dtype=np.float64).reshape(-1, 5)
        dih = self.dihedrals
        p14 = [(d[0], d[3]) for d in dih if d[7]]
        return {
            "atomCount": n,
            "charges": np.array(self.charges), "masses": np.array(self.masses),
            "atomicNumbers": np.array(self.z, dtype=np.int32),
            "atomTypes": np.array(self.types, dtype=np.int32), "typeCount": len(TYPE_ORDER),
            "ljA": lj_a, "ljB": lj_b,
            "residueNames": self.resnames, "residueOfAtom": np.array(self.res, dtype=np.int32),
            "bonds": {"count": len(bonds), "atomA": bonds[:, 0].astype(np.int32),
                      "atomB": bonds[:, 1].astype(np.int32), "k": bonds[:, 2] * BOND_K_SCALE,
                      "r0": bonds[:, 3].copy()},
            "angles": {"count": len(angles), "atomA": angles[:, 0].astype(np.int32),
                       "atomB": angles[:, 1].astype(np.int32), "atomC": angles[:, 2].astype(np.int32),
                       "k": angles[:, 3] * ANGLE_K_SCALE, "theta0": angles[:, 4].copy()},
            "dihedrals": {
                "count": len(dih),
                "atomA": np.array([d[0] for d in dih], dtype=np.int32),
                "atomB": np.array([d[1] for d in dih], dtype=np.int32),
                "atomC": np.array([d[2] for d in dih], dtype=np.int32),
                "atomD": np.array([d[3] for d in dih], dtype=np.int32),
                "k": np.array([d[4] * ENERGY_SCALE for d in dih]),
                "periodicity": np.array([float(d[5]) for d in dih]),
                "phase": np.array([d[6] for d in dih]),
                "pairs14": {"count": len(p14), "atomA": np.array([p[0] for p in p14], dtype=np.int32),
                            "atomB": np.array([p[1] for p in p14], dtype=np.int32),
                            "scee": np.full(len(p14), 1.2), "scnb": np.full(len(p14), 2.0)},
            },
            "exclusions": {"start": excl_start, "partners": np.array(partners, dtype=np.int32)},
            "boxFromTopology": {"lengths": [box_length] * 3, "angles": [90.0, 90.0, 90.0]},
            "isPeriodic": True,
            "moleculeCount": self.nmol, "moleculeOfAtom": np.array(self.mol, dtype=np.int32),
        }


def _box_for(mass_amu, density):
    return (mass_amu * AMU_PER_NM3_TO_G_PER_CM3 / density) ** (1.0 / 3.0)


def _fill(builder, rng, box, n_water, ions, occupied, clearance=0.25):
    """Waters on a jittered cubic lattice, ions on free sites, away from `occupied`."""
    sites_needed = n_water + len(ions)
    n = int(math.ceil(sites_needed ** (1.0 / 3.0)))
    while True:
        spacing = box / n
        g = (np.arange(n) + 0.5) * spacing
        sites = np.array(np.meshgrid(g, g, g, indexing="ij")).reshape(3, -1).T
        if len(occupied):
            from scipy.spatial import cKDTree

            tree = cKDTree(np.mod(occupied, box), boxsize=box)
            nearest, _ = tree.query(np.mod(sites, box), k=1, distance_upper_bound=clearance * 1.0001)
            sites = sites[nearest > clearance]
        if len(sites) >= sites_needed:
            break
        n += 1
    order = rng.permutation(len(sites))[:sites_needed]
    chosen = sites[np.sort(order)]
    jitter = rng.uniform(-0.02, 0.02, size=chosen.shape)
    chosen = chosen + jitter
    rot = _random_rotations(rng, n_water)
    ion_slots = set(rng.choice(len(chosen), size=len(ions), replace=False).tolist()) if ions else set()
    w = 0
    ion_iter = iter(ions)
    for k, site in enumerate(chosen):
        if k in ion_slots:
            builder.add_ion(next(ion_iter), site)
        else:
            builder.add_water(site, rot[w])
            w += 1


def water_box(n_atoms: int, density: float = 0.997, seed: int = 0):
    """⌊n/3⌋ TIP3P waters plus Na+ (remainder 1) or Na+ and Cl- (remainder 2)."""
    rng = np.random.default_rng(seed)
    n_water = n_atoms // 3
    ions = {0: [], 1: ["NA"], 2: ["NA", "CL"]}[n_atoms - 3 * n_water]
    mass = n_water * sum(WATER_MASS) + sum(TYPES[i][0] for i in ions)
    box = _box_for(mass, density)
    b = _Builder()
    _fill(b, rng, box, n_water, ions, np.zeros((0, 3)))
    return b.topology(box), np.array(b.pos).reshape(-1)


def solvated_chain(n_atoms: int, chain_atoms: int, density: float = 0.997, seed: int = 0,
                   box_length: float | None = None):
    """A chain solute (net -1) with one Na+ in TIP3P water; total exactly n_atoms when
    n_atoms - chain_atoms - 1 is a multiple of 3, otherwise the nearest smaller count."""
    rng = np.random.default_rng(seed)
    n_water = (n_atoms - chain_atoms - 1) // 3
    mass = n_water * sum(WATER_MASS) + chain_atoms * TYPES["C"][0] + TYPES["NA"][0]
    box = box_length if box_length is not None else _box_for(mass, density)
    b = _Builder()
    chain, lengths = _chain(rng, chain_atoms, box)
    chain = chain + box / 2
    b.add_chain(rng, chain, lengths)
    _fill(b, rng, box, n_water, ["NA"], chain, clearance=0.3)
    return b.topology(box), np.array(b.pos).reshape(-1)


def config0(seed: int = 0):
    """1190 atoms: 22-atom chain, 1 Na+, 389 TIP3P waters in a 22.65 Å cube."""
    return solvated_chain(1190, 22, seed=seed, box_length=2.265)


def batch(count: int = 64, low: int = 1000, high: int = 12000, seed: int = 0,
          chain_low: int = 20, chain_high: int = 400):
    """Uneven solvated systems: sizes log-uniform in [low, high], chains of 20-400 atoms."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(low), math.log(high), size=count)).astype(int)
    out = []
    for k, size in enumerate(sizes):
        chain = int(rng.integers(chain_low, min(chain_high, max(chain_low + 1, size // 5)) + 1))
        out.append(solvated_chain(int(size), chain, seed=seed * 1000 + k))
    return out
