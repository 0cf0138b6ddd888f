"""The trajectory writers' oracle, pinned to the reference's own writer tests
(test/physics.test.js:253-376, test/interface.test.js:443-510) and to ECMAScript's number
formatting, plus the library's host-side DCD header against it (no GPU needed).
"""
import ctypes as C
import math
import struct

import numpy as np
import pytest

from goldens import system_for
from oracle import traj as ot
from rainmd_b200 import _lib as L
from rainmd_b200.amber import parse_inpcrd


@pytest.mark.parametrize("x,digits,text", [
    (0.00390625, 7, "0.0039063"),   # an exact binary tie: the larger n (printf's half-even gives ...62)
    (-0.00390625, 7, "-0.0039063"),
    (-1e-9, 7, "-0.0000000"),       # the sign survives a value that rounds to zero
    (-0.0, 7, "0.0000000"),         # -0 is not below zero
    (123.456, 7, "123.4560000"),
    (1.005, 2, "1.00"),             # 1.005 is 1.00499999999999989... in binary
    (1.45, 1, "1.4"),
    (0.5, 0, "1"), (2.5, 0, "3"), (-0.5, 0, "-1"),
])
def test_to_fixed_follows_ecmascript(x, digits, text):
    assert ot.to_fixed(x, digits) == text


@pytest.mark.parametrize("x,text", [
    (1.5, "1.5000000e+0"), (0.0, "0.0000000e+0"), (20.0, "2.0000000e+1"),
    (2.44140625e-4, "2.4414063e-4"),  # exact tie, rounded up
    (1e-7, "1.0000000e-7"), (9.99999995, "9.9999999e+0"), (123456.789, "1.2345679e+5"),
])
def test_to_exponential_follows_ecmascript(x, text):
    assert ot.to_exponential(x, 7) == text


def test_dcd_header_and_cell_layout():
    """physics.test.js:253-285: the header fields and the cell order OpenMM writes."""
    box = [2.5, 0, 0, 0.3, 2.6, 0, 0.4, 0.5, 2.7]
    header = ot.dcd_header(3, 2, 0, 5, 0.002, True, "Created by RainMD", "Created X")
    assert struct.unpack_from("<i", header, 0)[0] == 84
    assert header[4:8] == b"CORD"
    assert struct.unpack_from("<i", header, 8)[0] == 2
    assert struct.unpack_from("<i", header, 16)[0] == 5
    assert struct.unpack_from("<i", header, 20)[0] == 5
    assert abs(struct.unpack_from("<f", header, 44)[0] - 0.002 / 0.04888821) < 1e-6
    assert struct.unpack_from("<i", header, 48)[0] == 1
    assert struct.unpack_from("<i", header, 84)[0] == 24
    assert struct.unpack_from("<i", header, 268)[0] == 3
    cell = ot.cell_from_vectors(box)
    assert abs(cell[0] - 25) < 1e-9
    assert abs(cell[2] - math.hypot(0.3, 2.6) * 10) < 1e-9
    assert abs(cell[5] - math.hypot(0.4, 0.5, 2.7) * 10) < 1e-9
    assert abs(cell[1] - 0.3 * 2.5 / (2.5 * math.hypot(0.3, 2.6))) < 1e-12
    # the frame: the cell record, then x, y and z records in angstroms
    positions = [0, 0, 0, 0.1, 0.2, 0.3, -0.4, 0.5, -0.6]
    frame = ot.dcd_frame(positions, box, periodic=True, image=False)
    assert len(frame) == 56 + 3 * (4 * 3 + 8)
    assert struct.unpack_from("<i", frame, 0)[0] == 48 and struct.unpack_from("<i", frame, 52)[0] == 48
    x = struct.unpack_from("<ifffi", frame, 56)
    assert x[0] == 12 and x[4] == 12 and np.allclose(x[1:4], [0, 1, -4])


def test_library_dcd_header_is_the_oracle_header():
    lib = L.load()
    out = np.zeros(276, np.uint8)
    assert lib.rmd_dcd_header(3, 2, 7, 5, 0.002, 1, b"RainMD ala-wat", b"Created 2026-01-01T00:00:00.000Z",
                              out.ctypes.data_as(C.c_void_p)) == 0
    assert out.tobytes() == ot.dcd_header(3, 2, 7, 5, 0.002, True, "RainMD ala-wat",
                                          "Created 2026-01-01T00:00:00.000Z")
    assert lib.rmd_dcd_frame_bytes(1190, 1) == 56 + 3 * (4 * 1190 + 8)
    assert lib.rmd_dcd_frame_bytes(1190, 0) == 3 * (4 * 1190 + 8)


def test_a_nan_frame_is_refused():
    with pytest.raises(ValueError, match="no longer a number"):
        ot.dcd_frame([0, 0, 0, 1, float("nan"), 1], None, periodic=False, image=False)


def test_restart_round_trips_through_the_reader():
    """physics.test.js:293-317 with this package's inpcrd reader."""
    s, pos, _ = system_for("ala-wat")
    velocities = np.sin(np.arange(pos.size) * 0.7) * 0.5
    box = ot.box_from_vectors(s["boxVectors"])
    text = ot.restart_text(pos, velocities, box, time=1.5)
    again = parse_inpcrd(text, expected_atom_count=len(pos) // 3)
    assert again["time"] == 1.5
    assert np.max(np.abs(again["positions"] - pos.reshape(-1))) < 1e-7
    assert np.max(np.abs(again["velocities"] - velocities)) < 1e-6
    for axis in range(3):
        assert abs(again["box"]["lengths"][axis] - box["lengths"][axis]) < 1e-7


def test_restart_refuses_wide_and_non_finite_values():
    """physics.test.js:319-357: the first failing value decides."""
    with pytest.raises(OverflowError, match="12-column"):
        ot.restart_text([1e6, 0, 0])
    with pytest.raises(ValueError, match="no longer a number"):
        ot.restart_text([1, float("nan"), 0])
    with pytest.raises(ValueError, match="no longer a number"):
        ot.restart_text([1, 2, 3], velocities=[0, float("inf"), 0])
    assert ot.restart_text([1, 2, 3]).startswith("RainMD restart\n")


def test_imaging_keeps_molecules_whole():
    """interface.test.js:443-510 on ala-wat: three molecules pushed out by whole box
    vectors come back with every centroid in the cell and every bond intact; an in-cell
    structure does not move."""
    s, pos, _ = system_for("ala-wat")
    box = np.asarray(s["boxVectors"], np.float64)
    t = s["topology"]
    mol = np.asarray(t["moleculeOfAtom"])
    drifted = pos.reshape(-1, 3).astype(np.float64).copy()
    moved = np.isin(mol, [1, 2, 3])
    drifted[moved, 0] += box[0] * 2
    drifted[moved, 1] -= box[4]
    drifted[moved, 2] += box[8] * 3
    wrapped = ot.image_molecules(drifted, box, mol, t["moleculeCount"]).reshape(-1, 3)
    for m in range(t["moleculeCount"]):
        c = wrapped[mol == m].mean(0)
        assert -1e-9 <= c[2] < box[8] + 1e-9 and -1e-9 <= c[1] < box[4] + 1e-9 and -1e-9 <= c[0] < box[0] + 1e-9
    a, b = np.asarray(t["bonds"]["atomA"]), np.asarray(t["bonds"]["atomB"])
    assert np.max(np.linalg.norm(wrapped[a] - wrapped[b], axis=1)) < 0.25
    inside = ot.image_molecules(pos, box, mol, t["moleculeCount"])
    assert np.max(np.abs(inside - pos.reshape(-1))) < 1e-12
