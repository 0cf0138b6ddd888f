"""CPU oracle of the trajectory writers: test infrastructure only (it checks
rainmd_b200/csrc/traj.cu; nothing in the product imports it).

Restates, in Python floats (IEEE float64, the JavaScript Number) and exact decimal arithmetic:
  imageMolecules       shared/traj/imaging.js:39-91
  cellFromVectors      shared/traj/dcd.js:214-230 (Math.hypot as the Kahan-compensated scaled
                       sum of squares an ECMAScript engine evaluates)
  DcdWriter frame and header bytes   shared/traj/dcd.js:96-200
  writeRestart         shared/traj/rst7.js:20-101 (toFixed / toExponential per ECMAScript:
                       the exact binary value rounded, the larger magnitude on a tie)
  boxFromVectors       web/app.js:326-343
and is pinned by the reference's own writer tests (test/physics.test.js:253-376,
test/interface.test.js:443-510), restated in tests/test_traj_oracle.py.
"""
from __future__ import annotations

import math
import struct
from decimal import ROUND_HALF_UP, Decimal, localcontext

import numpy as np

AKMA_PICOSECONDS = 0.04888821
ANGSTROM_PER_NM = 10
NM_PER_ANGSTROM = 0.1
AMBER_VELOCITY_SCALE = 20.455


def image_molecules(positions, box, molecule_of_atom, count):
    """imaging.js:39-91. `positions` are the values the writer is handed (f32 from the device
    widened to float64); the sums run in atom order as the reference's single pass does."""
    p = [float(v) for v in np.asarray(positions, dtype=np.float64).reshape(-1)]
    n = len(p) // 3
    out = list(p)
    if box is None:
        return np.array(out)
    ax, _, _, bx, by, _, cx, cy, cz = (float(v) for v in box)
    if not (ax > 0) or not (by > 0) or not (cz > 0):
        return np.array(out)
    sums = [0.0] * (3 * count)
    sizes = [0.0] * count
    mol = [int(m) for m in molecule_of_atom]
    for atom in range(n):
        m = mol[atom]
        sums[3 * m] += p[3 * atom]
        sums[3 * m + 1] += p[3 * atom + 1]
        sums[3 * m + 2] += p[3 * atom + 2]
        sizes[m] += 1
    shifts = [0.0] * (3 * count)
    for m in range(count):
        size = sizes[m]
        if size == 0:
            continue
        x, y, z = sums[3 * m] / size, sums[3 * m + 1] / size, sums[3 * m + 2] / size
        nc = float(np.floor(z / cz))  # a float floor keeps -0.0, as Math.floor does
        y_c = y - nc * cy
        nb = float(np.floor(y_c / by))
        x_cb = x - nc * cx - nb * bx
        na = float(np.floor(x_cb / ax))
        shifts[3 * m] = -(na * ax + nb * bx + nc * cx)
        shifts[3 * m + 1] = -(nb * by + nc * cy)
        shifts[3 * m + 2] = -(nc * cz)
    for atom in range(n):
        m = mol[atom]
        for c in range(3):
            out[3 * atom + c] = p[3 * atom + c] + shifts[3 * m + c]
    return np.array(out)


def script_hypot(*values):
    """Math.hypot: scaled by the largest magnitude, Kahan-compensated sum of squares."""
    v = [abs(float(x)) for x in values]
    top = max(v) if v else 0.0
    if top == 0.0:
        return 0.0
    total = carry = 0.0
    for a in v:
        n = a / top
        term = n * n - carry
        nxt = total + term
        carry = (nxt - total) - term
        total = nxt
    return math.sqrt(total) * top


def cell_from_vectors(v):
    a, b, c = [float(x) for x in v[0:3]], [float(x) for x in v[3:6]], [float(x) for x in v[6:9]]
    la, lb, lc = script_hypot(*a), script_hypot(*b), script_hypot(*c)

    def dot(u, w):
        return u[0] * w[0] + u[1] * w[1] + u[2] * w[2]

    cos_alpha = dot(b, c) / (lb * lc) if lb * lc > 0 else 0.0
    cos_beta = dot(a, c) / (la * lc) if la * lc > 0 else 0.0
    cos_gamma = dot(a, b) / (la * lb) if la * lb > 0 else 0.0
    return [la * ANGSTROM_PER_NM, cos_gamma, lb * ANGSTROM_PER_NM, cos_beta, cos_alpha, lc * ANGSTROM_PER_NM]


def dcd_frame(positions, box, molecule_of_atom=None, count=0, periodic=True, image=True):
    """One frame's bytes (dcd.js:96-161). Raises ValueError on a non-finite coordinate."""
    p = np.asarray(positions, dtype=np.float64).reshape(-1)
    if not np.all(np.isfinite(p)):
        raise ValueError("a coordinate handed to the DCD writer is no longer a number")
    n = len(p) // 3
    coords = image_molecules(p, box, molecule_of_atom, count) if image and molecule_of_atom is not None else p
    xyz = coords.reshape(-1, 3)
    out = b""
    if periodic:
        out += struct.pack("<i", 48) + struct.pack("<6d", *cell_from_vectors(box)) + struct.pack("<i", 48)
    for axis in range(3):
        values = (xyz[:, axis] * ANGSTROM_PER_NM).astype(np.float32)
        out += struct.pack("<i", 4 * n) + values.astype("<f4").tobytes() + struct.pack("<i", 4 * n)
    return out


def dcd_header(atom_count, frames, first_step, interval, timestep, periodic, title, created):
    h = bytearray(276)
    struct.pack_into("<i", h, 0, 84)
    h[4:8] = b"CORD"
    struct.pack_into("<iiii", h, 8, frames, first_step, interval, max(0, frames - 1) * interval)
    struct.pack_into("<f", h, 44, timestep / AKMA_PICOSECONDS)
    struct.pack_into("<i", h, 48, 1 if periodic else 0)
    struct.pack_into("<iiii", h, 84, 24, 84, 164, 2)
    for offset, text in ((100, title), (180, created)):
        for k, ch in enumerate(text[:80]):
            h[offset + k] = ord(ch) if ord(ch) < 128 else 0x3F
    struct.pack_into("<iiii", h, 260, 164, 4, atom_count, 4)
    return bytes(h)


def to_fixed(x: float, digits: int = 7) -> str:
    """Number.prototype.toFixed for |x| < 1e21."""
    x = float(x)
    if x != x:
        return "NaN"
    sign = "-" if x < 0 else ""
    with localcontext() as ctx:
        ctx.prec = 2000  # every operation below is exact
        q = Decimal(abs(x)).quantize(Decimal(1).scaleb(-digits), rounding=ROUND_HALF_UP)
        text = format(q, "f")
    return sign + text


def to_exponential(x: float, digits: int = 7) -> str:
    """Number.prototype.toExponential(digits) for finite x."""
    x = float(x)
    if x == 0:
        return "0." + "0" * digits + "e+0" if digits else "0e+0"
    sign = "-" if x < 0 else ""
    with localcontext() as ctx:
        ctx.prec = 2000  # every operation below is exact
        d = Decimal(abs(x))
        e = d.adjusted()
        q = d.scaleb(-e).quantize(Decimal(1).scaleb(-digits), rounding=ROUND_HALF_UP)
        if q >= 10:
            e += 1
            q = d.scaleb(-e).quantize(Decimal(1).scaleb(-digits), rounding=ROUND_HALF_UP)
        mant = format(q, "f")
    return f"{sign}{mant}e{'-' if e < 0 else '+'}{abs(e)}"


def _columns(values):
    lines = []
    for start in range(0, len(values), 6):
        line = ""
        for v in values[start:start + 6]:
            if not math.isfinite(v):
                raise ValueError("a coordinate handed to the restart writer is no longer a number")
            text = to_fixed(v, 7)
            if len(text) > 12:
                raise OverflowError(f"coordinate {v} does not fit the 12-column restart format")
            line += text.rjust(12)
        lines.append(line)
    return lines


def box_from_vectors(v):
    a, b, c = [float(x) for x in v[0:3]], [float(x) for x in v[3:6]], [float(x) for x in v[6:9]]
    la, lb, lc = script_hypot(*a), script_hypot(*b), script_hypot(*c)

    def dot(u, w):
        return u[0] * w[0] + u[1] * w[1] + u[2] * w[2]

    def degrees(value):
        return (math.acos(max(-1.0, min(1.0, value))) * 180) / math.pi

    return {"lengths": [la, lb, lc],
            "angles": [degrees(dot(b, c) / (lb * lc)), degrees(dot(a, c) / (la * lc)),
                       degrees(dot(a, b) / (la * lb))]}


def restart_text(positions, velocities=None, box=None, time=0.0, title="RainMD restart"):
    """writeRestart (rst7.js:63-101); `box` is {lengths (nm), angles (degrees)}."""
    p = [float(v) for v in np.asarray(positions, dtype=np.float64).reshape(-1)]
    n = len(p) // 3
    lines = [title, f"{str(n).rjust(5)}{to_exponential(time, 7).rjust(15)}"]
    lines += _columns([v / NM_PER_ANGSTROM for v in p])
    if velocities is not None:
        unit = AMBER_VELOCITY_SCALE * NM_PER_ANGSTROM
        lines += _columns([float(v) / unit for v in np.asarray(velocities, dtype=np.float64).reshape(-1)])
    if box is not None:
        L, A = box["lengths"], box["angles"]
        lines += _columns([L[0] / NM_PER_ANGSTROM, L[1] / NM_PER_ANGSTROM, L[2] / NM_PER_ANGSTROM,
                           A[0], A[1], A[2]])
    return "\n".join(lines) + "\n"
