"""Regenerate the golden fixtures under tests/golden/ from RainMD's own test fixtures.

RainMD ships AMBER systems (`test/fixtures/*.prmtop`, `*.inpcrd`) and OpenMM 8.4
Reference-platform single-point dumps of them (`test/fixtures/*.json`, produced by the
reference's `tools/oracle/dump_openmm_reference.py`). This script parses the AMBER files
with this package's own reader and stores, per case, the parsed topology arrays, the
coordinates, the box, and the OpenMM energies and forces as one compressed `.npz`, so the
tests and the GPU box never need the reference tree.

Run from the repository root:  python tests/golden/make_golden.py <root of a RainMD checkout>
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from rainmd_b200.amber import parse_inpcrd, parse_prmtop  # noqa: E402


def flatten(prefix: str, value, out: dict):
    if isinstance(value, dict):
        for key, item in value.items():
            flatten(f"{prefix}{key}.", item, out)
        return
    key = prefix[:-1]
    if value is None:
        return
    if isinstance(value, (list, tuple)) and value and isinstance(value[0], str):
        out[key] = np.array(value)
    else:
        out[key] = np.asarray(value)


def save_system(root: str, name: str, out: dict):
    fixtures = os.path.join(root, "test", "fixtures")
    with open(os.path.join(fixtures, f"{name}.prmtop")) as handle:
        topology = parse_prmtop(handle.read())
    with open(os.path.join(fixtures, f"{name}.inpcrd")) as handle:
        coordinates = parse_inpcrd(handle.read(), topology["atomCount"])
    flatten("topology.", topology, out)
    out["positions"] = coordinates["positions"]
    if coordinates["box"] is not None:
        out["box.lengths"] = np.array(coordinates["box"]["lengths"])
        out["box.angles"] = np.array(coordinates["box"]["angles"])


def save_dump(root: str, dump: str, prefix: str, out: dict, forces: bool):
    with open(os.path.join(root, "test", "fixtures", f"{dump}.json")) as handle:
        data = json.load(handle)
    energy = data["energy"]
    for key in ("total", "ljOnly", "coulombOnly"):
        out[f"{prefix}energy.{key}"] = np.float64(energy[key])
    for key, value in energy["byForceGroup"].items():
        label = key.split(":", 1)[1]
        out[f"{prefix}group.{label}"] = np.float64(value["energy"])
    if data.get("pme") and data["pme"].get("alpha") is not None:
        out[f"{prefix}pme.alpha"] = np.float64(data["pme"]["alpha"])
        out[f"{prefix}pme.grid"] = np.array(data["pme"]["grid"], dtype=np.int32)
    out[f"{prefix}inputs.constraints"] = np.array(str(data["inputs"]["constraints"]))
    out[f"{prefix}inputs.dispersion"] = np.array(bool(data["inputs"].get("dispersionCorrection")))
    if data["inputs"].get("volumeScale") is not None:
        out[f"{prefix}inputs.volumeScale"] = np.float64(data["inputs"]["volumeScale"])
    if forces and "forces" in data:
        for key in ("total", "ljOnly", "coulombOnly"):
            out[f"{prefix}forces.{key}"] = np.array(data["forces"][key], dtype=np.float64)
    if "positions" in data:
        out[f"{prefix}positions"] = np.array(data["positions"], dtype=np.float64)
    if data.get("restraint") and data["restraint"]["atomCount"] > 0:
        out[f"{prefix}restraint.force"] = np.float64(data["restraint"]["force"])
        out[f"{prefix}restraint.atoms"] = np.array(data["restraint"]["atoms"], dtype=np.int32)
    out[f"{prefix}exceptionCount"] = np.int64(data["exceptionCount"])
    out[f"{prefix}constraintCount"] = np.int64(data["constraintCount"])


def main():
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py <root of a RainMD checkout>")
    root = sys.argv[1]
    cases = {
        "ala-vac": [("ala-vac-nocutoff", True)],
        "ala-wat": [("ala-wat-pme", True), ("ala-wat-pme-free", True), ("ala-wat-pme-tail", False),
                    ("ala-wat-ewald", False), ("ala-wat-scale-0.97", False),
                    ("ala-wat-scale-1.00", False), ("ala-wat-scale-1.02", False),
                    ("ala-wat-restraint-500", True)],
        "ala-oct": [("ala-oct-pme", True)],
        "ala-wat-big": [],
    }
    for system, dumps in cases.items():
        out: dict = {}
        save_system(root, system, out)
        for dump, forces in dumps:
            save_dump(root, dump, f"{dump}:", out, forces)
        path = os.path.join(HERE, f"{system}.npz")
        np.savez_compressed(path, **out)
        print(f"wrote {path} ({os.path.getsize(path)} bytes, {len(out)} arrays)")


if __name__ == "__main__":
    main()
