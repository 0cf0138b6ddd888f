"""AMBER parm7 / inpcrd reading into the topology dictionary the system builder takes.

This is the host-side ingestion that sits upstream of the engine boundary, restated
from RainMD's `shared/amber/sections.js` (Fortran-format section reader),
`shared/amber/prmtop.js:111-395` (`parsePrmtop`) and `shared/amber/inpcrd.js:34-196`
(`parseInpcrd`, `boxVectorsFromLengthsAndAngles`). Units are converted once, at parse
time, into nm, kJ/mol, ps, amu and e (`shared/units.js`).

Only what the MD path reads is kept; the flag audit and UI-facing fields of the
reference parser are out of scope.
"""
from __future__ import annotations

import math
import re

import numpy as np

# shared/units.js
KCAL_TO_KJ = 4.184
NM_PER_ANGSTROM = 0.1
AMBER_VELOCITY_SCALE = 20.455  # angstroms per AMBER time unit -> per ps (units.js:44)
AMBER_CHARGE_SCALE = 18.2223
ENERGY_SCALE = KCAL_TO_KJ
BOND_K_SCALE = 2 * KCAL_TO_KJ / (NM_PER_ANGSTROM * NM_PER_ANGSTROM)
ANGLE_K_SCALE = 2 * KCAL_TO_KJ

POINTER_NAMES = [
    "NATOM", "NTYPES", "NBONH", "MBONA", "NTHETH", "MTHETA", "NPHIH", "MPHIA",
    "NHPARM", "NPARM", "NNB", "NRES", "NBONA", "NTHETA", "NPHIA", "NUMBND",
    "NUMANG", "NPTRA", "NATYP", "NPHB", "IFPERT", "NBPER", "NGPER", "NDPER",
    "MBPER", "MGPER", "MDPER", "IFBOX", "NMXRS", "IFCAP", "NUMEXTRA", "NCOPY",
]
DEFAULT_SCEE = 1.2
DEFAULT_SCNB = 2.0

_FORMAT = re.compile(r"^\s*(\d*)\s*([aAiIeEfFgG])\s*(\d+)(?:\.(\d+))?\s*$")


def _read_sections(text: str) -> dict:
    """Fortran fixed-width %FLAG sections (shared/amber/sections.js:60-147)."""
    sections: dict = {}
    flag = None
    fmt = None
    values: list = []

    def commit():
        if flag is not None and fmt is not None:
            sections[flag] = values

    for line in text.splitlines():
        if line.startswith("%VERSION") or line.startswith("%COMMENT"):
            continue
        if line.startswith("%FLAG"):
            commit()
            flag = line[5:].strip()
            fmt = None
            values = []
            continue
        if line.startswith("%FORMAT"):
            inner = line[line.index("(") + 1: line.rindex(")")]
            m = _FORMAT.match(inner)
            if m is None:
                raise ValueError(f"unsupported AMBER %FORMAT descriptor: {inner!r}")
            per_line = int(m.group(1)) if m.group(1) else 1
            letter = m.group(2).lower()
            kind = "string" if letter == "a" else ("integer" if letter == "i" else "float")
            fmt = (per_line, kind, int(m.group(3)))
            continue
        if flag is None or fmt is None:
            continue
        per_line, kind, width = fmt
        for index in range(per_line):
            start = index * width
            if start >= len(line):
                break
            field = line[start:start + width]
            if kind == "string":
                values.append(field)
                continue
            trimmed = field.strip()
            if not trimmed:
                continue
            values.append(float(trimmed) if kind == "float" else int(trimmed))
    commit()
    return sections


def _lj_to_internal(a_kcal_a12: float, b_kcal_a6: float) -> tuple[float, float]:
    """shared/units.js:100-107 (`ljCoefficientsToInternal`)."""
    return (a_kcal_a12 * ENERGY_SCALE * NM_PER_ANGSTROM ** 12,
            b_kcal_a6 * ENERGY_SCALE * NM_PER_ANGSTROM ** 6)


def _molecules(atom_count: int, bond_a: np.ndarray, bond_b: np.ndarray):
    """Connected components over bonds, numbered by first atom (prmtop.js:66-103)."""
    parent = list(range(atom_count))

    def find(node):
        root = node
        while parent[root] != root:
            root = parent[root]
        while parent[node] != root:
            parent[node], node = root, parent[node]
        return root

    for a, b in zip(bond_a.tolist(), bond_b.tolist()):
        ra, rb = find(a), find(b)
        if ra != rb:
            parent[rb] = ra
    root_to_molecule: dict = {}
    molecule_of_atom = np.zeros(atom_count, dtype=np.int32)
    for atom in range(atom_count):
        root = find(atom)
        molecule = root_to_molecule.setdefault(root, len(root_to_molecule))
        molecule_of_atom[atom] = molecule
    return len(root_to_molecule), molecule_of_atom


def parse_prmtop(text: str) -> dict:
    """Parse a parm7 topology into internal units (prmtop.js:111-395)."""
    sections = _read_sections(text)
    if "POINTERS" not in sections:
        raise ValueError("not an AMBER parm7 topology: no %FLAG POINTERS")
    pointers = {name: (sections["POINTERS"][i] if i < len(sections["POINTERS"]) else 0)
                for i, name in enumerate(POINTER_NAMES)}
    n = pointers["NATOM"]
    if pointers.get("NUMEXTRA", 0) > 0:
        raise ValueError("extra points (NUMEXTRA > 0) are not supported")

    def req(flag):
        if flag not in sections:
            raise ValueError(f"AMBER topology is missing required %FLAG {flag}")
        return sections[flag]

    def opt(flag):
        return sections.get(flag, [])

    charges = np.array(req("CHARGE")[:n], dtype=np.float64) / AMBER_CHARGE_SCALE
    masses = np.array(req("MASS")[:n], dtype=np.float64)
    if "ATOMIC_NUMBER" in sections:
        atomic_numbers = np.array(sections["ATOMIC_NUMBER"][:n], dtype=np.int32)
    else:
        atomic_numbers = np.where((masses > 0) & (masses < 3.5), 1, 0).astype(np.int32)
    atom_types = np.array(req("ATOM_TYPE_INDEX")[:n], dtype=np.int32) - 1
    nres = pointers["NRES"]
    residue_names = [str(v).strip() for v in req("RESIDUE_LABEL")[:nres]]
    residue_first = np.array(req("RESIDUE_POINTER")[:nres], dtype=np.int32) - 1
    residue_of_atom = np.zeros(n, dtype=np.int32)
    for r in range(nres):
        end = residue_first[r + 1] if r + 1 < nres else n
        residue_of_atom[residue_first[r]:end] = r

    ntypes = pointers["NTYPES"]
    nb_index = req("NONBONDED_PARM_INDEX")
    raw_a = req("LENNARD_JONES_ACOEF")
    raw_b = req("LENNARD_JONES_BCOEF")
    lj_a = np.zeros(ntypes * ntypes)
    lj_b = np.zeros(ntypes * ntypes)
    for i in range(ntypes):
        for j in range(ntypes):
            p = nb_index[ntypes * i + j]
            if p > 0:
                lj_a[ntypes * i + j], lj_b[ntypes * i + j] = _lj_to_internal(raw_a[p - 1], raw_b[p - 1])
            elif p < 0:
                raise ValueError("10-12 hydrogen-bond LJ terms are not supported")

    def stride(v):
        return abs(v) // 3

    bond_k_table = req("BOND_FORCE_CONSTANT")
    bond_r0_table = req("BOND_EQUIL_VALUE")
    raw = list(opt("BONDS_INC_HYDROGEN")) + list(opt("BONDS_WITHOUT_HYDROGEN"))
    nb = len(raw) // 3
    bonds = {
        "count": nb,
        "atomA": np.array([stride(raw[3 * i]) for i in range(nb)], dtype=np.int32),
        "atomB": np.array([stride(raw[3 * i + 1]) for i in range(nb)], dtype=np.int32),
        "k": np.array([bond_k_table[raw[3 * i + 2] - 1] * BOND_K_SCALE for i in range(nb)]),
        "r0": np.array([bond_r0_table[raw[3 * i + 2] - 1] * NM_PER_ANGSTROM for i in range(nb)]),
    }

    angle_k_table = req("ANGLE_FORCE_CONSTANT")
    angle_t_table = req("ANGLE_EQUIL_VALUE")
    raw = list(opt("ANGLES_INC_HYDROGEN")) + list(opt("ANGLES_WITHOUT_HYDROGEN"))
    na = len(raw) // 4
    angles = {
        "count": na,
        "atomA": np.array([stride(raw[4 * i]) for i in range(na)], dtype=np.int32),
        "atomB": np.array([stride(raw[4 * i + 1]) for i in range(na)], dtype=np.int32),
        "atomC": np.array([stride(raw[4 * i + 2]) for i in range(na)], dtype=np.int32),
        "k": np.array([angle_k_table[raw[4 * i + 3] - 1] * ANGLE_K_SCALE for i in range(na)]),
        "theta0": np.array([angle_t_table[raw[4 * i + 3] - 1] for i in range(na)]),
    }

    dk = req("DIHEDRAL_FORCE_CONSTANT")
    dn = req("DIHEDRAL_PERIODICITY")
    dp = req("DIHEDRAL_PHASE")
    scee = sections.get("SCEE_SCALE_FACTOR")
    scnb = sections.get("SCNB_SCALE_FACTOR")
    raw = list(opt("DIHEDRALS_INC_HYDROGEN")) + list(opt("DIHEDRALS_WITHOUT_HYDROGEN"))
    nd = len(raw) // 5
    d_atoms = np.zeros((nd, 4), dtype=np.int32)
    d_k = np.zeros(nd)
    d_n = np.zeros(nd)
    d_phase = np.zeros(nd)
    p14a, p14b, p14scee, p14scnb = [], [], [], []
    seen = set()
    for i in range(nd):
        rc, rd = raw[5 * i + 2], raw[5 * i + 3]
        a, b, c, d = (stride(raw[5 * i]), stride(raw[5 * i + 1]), stride(rc), stride(rd))
        p = raw[5 * i + 4] - 1
        d_atoms[i] = (a, b, c, d)
        d_k[i] = dk[p] * ENERGY_SCALE
        d_n[i] = abs(dn[p])
        d_phase[i] = dp[p]
        if rc < 0 or rd < 0:
            continue
        lo, hi = min(a, d), max(a, d)
        if (lo, hi) in seen:
            continue
        seen.add((lo, hi))
        p14a.append(lo)
        p14b.append(hi)
        p14scee.append(DEFAULT_SCEE if scee is None else scee[p])
        p14scnb.append(DEFAULT_SCNB if scnb is None else scnb[p])
    dihedrals = {
        "count": nd,
        "atomA": d_atoms[:, 0].copy(), "atomB": d_atoms[:, 1].copy(),
        "atomC": d_atoms[:, 2].copy(), "atomD": d_atoms[:, 3].copy(),
        "k": d_k, "periodicity": d_n, "phase": d_phase,
        "pairs14": {
            "count": len(p14a),
            "atomA": np.array(p14a, dtype=np.int32), "atomB": np.array(p14b, dtype=np.int32),
            "scee": np.array(p14scee, dtype=np.float64), "scnb": np.array(p14scnb, dtype=np.float64),
        },
    }

    counts = req("NUMBER_EXCLUDED_ATOMS")
    listed = req("EXCLUDED_ATOMS_LIST")
    start = np.zeros(n + 1, dtype=np.int32)
    partners = []
    cursor = 0
    for atom in range(n):
        start[atom] = len(partners)
        for offset in range(counts[atom]):
            value = listed[cursor + offset]
            if value != 0:
                partners.append(value - 1)
        cursor += counts[atom]
    start[n] = len(partners)

    box_from_topology = None
    if pointers["IFBOX"] > 0 and "BOX_DIMENSIONS" in sections:
        bd = sections["BOX_DIMENSIONS"]
        box_from_topology = {"lengths": [bd[1] * 0.1, bd[2] * 0.1, bd[3] * 0.1],
                             "angles": [bd[0]] * 3}

    molecule_count, molecule_of_atom = _molecules(n, bonds["atomA"], bonds["atomB"])
    return {
        "atomCount": n, "charges": charges, "masses": masses, "atomicNumbers": atomic_numbers,
        "atomTypes": atom_types, "typeCount": ntypes, "ljA": lj_a, "ljB": lj_b,
        "residueNames": residue_names, "residueOfAtom": residue_of_atom,
        "bonds": bonds, "angles": angles, "dihedrals": dihedrals,
        "exclusions": {"start": start, "partners": np.array(partners, dtype=np.int32)},
        "boxFromTopology": box_from_topology, "isPeriodic": pointers["IFBOX"] > 0,
        "moleculeCount": molecule_count, "moleculeOfAtom": molecule_of_atom,
    }


def parse_inpcrd(text: str, expected_atom_count: int | None = None) -> dict:
    """ASCII inpcrd/rst7 in 12-column fields, Å → nm, velocities Å per AMBER time unit → nm/ps
    (inpcrd.js:34-130)."""
    lines = text.splitlines()
    title = lines[0].strip()
    header = lines[1].split()
    atom_count = int(header[0])
    time = float(header[1]) if len(header) > 1 else None
    if expected_atom_count is not None and expected_atom_count != atom_count:
        raise ValueError(f"coordinate file has {atom_count} atoms but the topology has "
                         f"{expected_atom_count}")
    numbers = []
    for line in lines[2:]:
        if not line.strip():
            continue
        for field in range(6):
            s = line[field * 12: field * 12 + 12].strip()
            if s:
                numbers.append(float(s))
    n3 = 3 * atom_count
    total = len(numbers)
    has_box = total in (n3 + 6, 2 * n3 + 6)
    has_vel = total in (2 * n3, 2 * n3 + 6)
    if total not in (n3, n3 + 6, 2 * n3, 2 * n3 + 6):
        raise ValueError(f"inpcrd holds {total} numbers for {atom_count} atoms")
    positions = np.array(numbers[:n3]) * NM_PER_ANGSTROM
    velocities = (np.array(numbers[n3:2 * n3]) * AMBER_VELOCITY_SCALE * NM_PER_ANGSTROM) if has_vel else None
    box = None
    if has_box:
        b = numbers[-6:]
        box = {"lengths": [b[0] * 0.1, b[1] * 0.1, b[2] * 0.1], "angles": [b[3], b[4], b[5]]}
    return {"title": title, "atomCount": atom_count, "time": time, "positions": positions,
            "velocities": velocities, "box": box}


def box_vectors_from_lengths_and_angles(box: dict) -> np.ndarray:
    """Reduced upper-triangular box vectors, row-major (inpcrd.js:154-196)."""
    a, b, c = box["lengths"]
    al, be, ga = (math.radians(x) for x in box["angles"])
    va = [a, 0.0, 0.0]
    vb = [b * math.cos(ga), b * math.sin(ga), 0.0]
    cx = c * math.cos(be)
    cy = c * (math.cos(al) - math.cos(be) * math.cos(ga)) / math.sin(ga)
    cz2 = c * c - cx * cx - cy * cy
    if cz2 <= 0:
        raise ValueError("box lengths and angles do not describe a realisable cell")
    vc = [cx, cy, math.sqrt(cz2)]
    for v in (va, vb, vc):
        for i in range(3):
            if abs(v[i]) < 1e-12 * a:
                v[i] = 0.0

    def js_round(x):
        return math.floor(x + 0.5)

    def reduce(target, source, comp):
        shift = js_round(target[comp] / source[comp])
        if shift != 0:
            for i in range(3):
                target[i] -= shift * source[i]

    reduce(vc, vb, 1)
    reduce(vc, va, 0)
    reduce(vb, va, 0)
    return np.array(va + vb + vc, dtype=np.float64)
