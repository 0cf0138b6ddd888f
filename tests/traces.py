"""Synthetic alpha-carbon traces for the ribbon tests (the reference's helix, strand and mixed
peptide fixtures are not part of this repository): an ideal alpha helix (2.3 A radius, 1.5 A
rise, 100 degrees a residue), a zig-zag beta strand (3.3 A repeat), and a chain of helix, coil
and strand, with optional chain breaks."""
import math

import numpy as np


def helix(n=24, origin=(0.0, 0.0, 0.0)):
    return np.array([[origin[0] + 0.23 * math.cos(math.radians(100 * i)),
                      origin[1] + 0.23 * math.sin(math.radians(100 * i)), origin[2] + 0.15 * i]
                     for i in range(n)])


def strand(n=24, origin=(0.0, 0.0, 0.0)):
    return np.array([[origin[0] + 0.33 * i, origin[1] + 0.1 * (-1) ** i, origin[2]] for i in range(n)])


def mixed():
    """10 helix, 6 coil, 8 strand residues in one chain."""
    h = helix(10)
    start = h[-1]
    coil = np.array([start + [0.3 * (k + 1), 0.15 * math.sin(k), 0.2 * math.cos(k)] for k in range(6)])
    s = strand(8, origin=tuple(coil[-1] + [0.35, 0.0, 0.0]))
    positions = np.vstack([h, coil, s])
    kinds = ["helix"] * 10 + ["coil"] * 6 + ["sheet"] * 8
    return positions, kinds
