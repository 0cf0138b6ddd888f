"""Topology → the "system" arrays a simulation runs, as RainMD's `buildSystem` does.

Restated from `shared/topology/system.js:40-235`. The three decisions that change the
energy are kept exactly: a constrained bond leaves the harmonic term, every excluded
pair becomes an exception (never a deletion), and a 1-4 pair is an exception scaled by
the SCEE/SCNB of the torsion that made it. Degrees of freedom are 3·N_massive −
constraints − 3 (`system.js:194-203`).

This code runs on the host, upstream of the engine boundary: the JavaScript page builds
the same dictionary and hands it to `GpuSimulation`, which is what `rmd_create` mirrors.
"""
from __future__ import annotations

import numpy as np

from .amber import box_vectors_from_lengths_and_angles

WATER_RESIDUES = {"WAT", "HOH", "H2O", "SOL", "TIP", "TP3", "SPC"}
ONE_4PI_EPS0 = 138.935456  # shared/units.js:47


def build_system(topology: dict, constraints: str = "HBonds", rigid_water: bool = True,
                 cutoff: float = 1.0, box=None, box_vectors=None) -> dict:
    """Return the system dictionary (system.js:40-235)."""
    if constraints not in ("none", "HBonds", "AllBonds"):
        raise ValueError(f"unsupported constraints mode {constraints!r}")
    n = topology["atomCount"]
    source = box if box is not None else topology.get("boxFromTopology")
    if box_vectors is not None:
        vectors = np.asarray(box_vectors, dtype=np.float64).copy()
    elif source is not None:
        vectors = box_vectors_from_lengths_and_angles(source)
    else:
        vectors = None
    if topology.get("isPeriodic") and vectors is None:
        raise ValueError("topology declares a periodic box but no box vectors were supplied")
    if vectors is not None:
        smallest = min(abs(vectors[0]), abs(vectors[4]), abs(vectors[8]))
        if cutoff > 0.5 * smallest:
            raise ValueError(f"a {cutoff} nm cutoff does not fit in a box whose smallest "
                             f"width is {smallest:.4f} nm")

    is_water = np.zeros(n, dtype=bool)
    if rigid_water:
        names = topology["residueNames"]
        for atom in range(n):
            if names[topology["residueOfAtom"][atom]] in WATER_RESIDUES:
                is_water[atom] = True
    bonds = topology["bonds"]
    z = topology["atomicNumbers"]
    ba, bb = bonds["atomA"], bonds["atomB"]
    constrained = np.zeros(bonds["count"], dtype=bool)
    for i in range(bonds["count"]):
        a, b = ba[i], bb[i]
        if constraints == "AllBonds":
            constrained[i] = True
        elif constraints == "HBonds" and (z[a] == 1 or z[b] == 1):
            constrained[i] = True
        if rigid_water and is_water[a] and is_water[b]:
            constrained[i] = True
    keep = ~constrained
    harmonic = {"count": int(keep.sum()), "atomA": ba[keep].astype(np.int32),
                "atomB": bb[keep].astype(np.int32), "k": bonds["k"][keep].copy(),
                "r0": bonds["r0"][keep].copy()}
    cons = {"count": int(constrained.sum()), "atomA": ba[constrained].astype(np.int32),
            "atomB": bb[constrained].astype(np.int32),
            "distance": bonds["r0"][constrained].copy()}

    pairs14 = topology["dihedrals"]["pairs14"]
    index14 = {(int(a), int(b)): i for i, (a, b) in enumerate(zip(pairs14["atomA"], pairs14["atomB"]))}
    ntypes = topology["typeCount"]
    q = topology["charges"]
    types = topology["atomTypes"]
    ex_a, ex_b, ex_q, ex_la, ex_lb = [], [], [], [], []
    start = topology["exclusions"]["start"]
    partners = topology["exclusions"]["partners"]
    for atom in range(n):
        for cursor in range(start[atom], start[atom + 1]):
            partner = int(partners[cursor])
            lo, hi = min(atom, partner), max(atom, partner)
            found = index14.get((lo, hi))
            tp = ntypes * types[atom] + types[partner]
            ex_a.append(lo)
            ex_b.append(hi)
            if found is None:
                ex_q.append(0.0)
                ex_la.append(0.0)
                ex_lb.append(0.0)
            else:
                ex_q.append(q[atom] * q[partner] / pairs14["scee"][found])
                ex_la.append(topology["ljA"][tp] / pairs14["scnb"][found])
                ex_lb.append(topology["ljB"][tp] / pairs14["scnb"][found])
    exceptions = {"count": len(ex_a), "atomA": np.array(ex_a, dtype=np.int32),
                  "atomB": np.array(ex_b, dtype=np.int32), "chargeProduct": np.array(ex_q),
                  "ljA": np.array(ex_la), "ljB": np.array(ex_lb)}

    mol = topology["moleculeOfAtom"]
    nmol = topology["moleculeCount"]
    counts = np.bincount(mol, minlength=nmol)
    mstart = np.zeros(nmol + 1, dtype=np.int32)
    mstart[1:] = np.cumsum(counts)
    matoms = np.argsort(mol, kind="stable").astype(np.int32)

    massive = int((topology["masses"] > 0).sum())
    dof = 3 * massive - cons["count"] - 3
    return {
        "topology": topology,
        "options": {"constraints": constraints, "rigidWater": rigid_water, "cutoff": cutoff},
        "boxVectors": vectors,
        "isPeriodic": vectors is not None,
        "harmonicBonds": harmonic,
        "constraints": cons,
        "exceptions": exceptions,
        "molecules": {"count": nmol, "start": mstart, "atoms": matoms},
        "degreesOfFreedom": dof,
    }
