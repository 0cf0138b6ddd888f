"""Loaders for the committed golden fixtures (tests/golden/*.npz).

Each fixture holds a parsed AMBER topology (from RainMD's `test/fixtures`), its
coordinates and box, and the OpenMM 8.4 Reference-platform single-point results RainMD
committed beside it. `tests/golden/make_golden.py` regenerates them.
"""
from __future__ import annotations

import os

import numpy as np

from rainmd_b200.topology import build_system

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name: str):
    """Return (topology, positions, box, raw) for a golden system."""
    data = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    raw = {k: data[k] for k in data.files}
    topo: dict = {}
    for key, value in raw.items():
        if not key.startswith("topology."):
            continue
        parts = key[len("topology."):].split(".")
        cursor = topo
        for part in parts[:-1]:
            cursor = cursor.setdefault(part, {})
        cursor[parts[-1]] = value
    for key in ("atomCount", "typeCount", "moleculeCount"):
        topo[key] = int(topo[key])
    for group in ("bonds", "angles", "dihedrals"):
        topo[group]["count"] = int(topo[group]["count"])
    topo["dihedrals"]["pairs14"]["count"] = int(topo["dihedrals"]["pairs14"]["count"])
    topo["residueNames"] = [str(x) for x in topo["residueNames"]]
    topo["isPeriodic"] = bool(topo["isPeriodic"])
    box = None
    if "box.lengths" in raw:
        box = {"lengths": raw["box.lengths"].tolist(), "angles": raw["box.angles"].tolist()}
    return topo, raw["positions"], box, raw


def system_for(name: str, constraints="HBonds", rigid_water=True, cutoff=1.0):
    topo, positions, box, raw = load(name)
    periodic = box is not None and cutoff > 0
    system = build_system(topo, constraints=constraints, rigid_water=rigid_water, cutoff=cutoff,
                          box=box if periodic else None)
    if not periodic:
        system["boxVectors"] = None
        system["isPeriodic"] = False
    return system, positions, raw
