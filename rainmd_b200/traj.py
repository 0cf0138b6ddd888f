"""Trajectory output from the device: the reference's DCD writer, AMBER restart writer and
molecule imaging (shared/traj/dcd.js, rst7.js, imaging.js) with the same names and options,
fed from the simulation's own position buffer instead of host arrays.

The reference page calls ``readPositions()`` and hands the array to ``DcdWriter.appendFrame``,
which images whole molecules and packs the frame on the host. Here ``appendFrame(simulation)``
has the device do both (rainmd_b200/csrc/traj.cu) and receives the finished frame bytes; the
file the writer produces is byte-identical to the reference's for the same coordinates and box.
"""
from __future__ import annotations

import ctypes as C
import datetime

import numpy as np

from . import _lib as L


def imageMolecules(simulation, index: int = 0) -> np.ndarray:
    """imaging.js:39-91 on the device: the current positions with every molecule translated
    by whole lattice vectors so that its centroid lies in the cell (FP64 nm, 3N)."""
    n = simulation.atom_counts[index]
    out = np.zeros(3 * n, np.float64)
    simulation._check(simulation._lib.rmd_image_molecules_at(
        simulation._h, index, out.ctypes.data_as(C.POINTER(C.c_double))))
    return out


class DcdWriter:
    """shared/traj/dcd.js:62-200. ``molecules`` is whether frames are imaged by molecule (the
    reference takes the partition itself; the device already holds it)."""

    def __init__(self, atomCount: int, timestep: float, interval: int, periodic: bool = False,
                 molecules: bool = True, firstStep: int = 0, title: str = "Created by RainMD"):
        self.atomCount = int(atomCount)
        self.timestep = float(timestep)
        self.interval = int(interval)
        self.periodic = bool(periodic)
        self.molecules = bool(molecules)
        self.firstStep = int(firstStep)
        self.title = title
        self.frameCount = 0
        self.chunks: list[bytes] = []
        self._lib = L.load()

    def appendFrame(self, simulation, index: int = 0) -> int:
        """Pack the simulation's current positions (and live box when periodic) as one frame.
        A non-finite coordinate raises NonFiniteStateError and the frames before it stay."""
        if simulation.atom_counts[index] != self.atomCount:
            raise ValueError(f"frame has {3 * simulation.atom_counts[index]} coordinates, "
                             f"expected {3 * self.atomCount}")
        size = self._lib.rmd_dcd_frame_bytes(self.atomCount, 1 if self.periodic else 0)
        frame = np.zeros(size, np.uint8)
        simulation._check(self._lib.rmd_dcd_frame_at(
            simulation._h, index, 1 if self.periodic else 0, 1 if self.molecules else 0,
            frame.ctypes.data_as(C.c_void_p)))
        self.chunks.append(frame.tobytes())
        self.frameCount += 1
        return self.frameCount

    def header(self, created: str | None = None) -> bytes:
        if created is None:
            created = "Created " + datetime.datetime.now(datetime.timezone.utc).isoformat(
                timespec="milliseconds").replace("+00:00", "Z")
        out = np.zeros(276, np.uint8)
        status = self._lib.rmd_dcd_header(self.atomCount, self.frameCount, self.firstStep, self.interval,
                                          self.timestep, 1 if self.periodic else 0, self.title.encode(),
                                          created.encode(), out.ctypes.data_as(C.c_void_p))
        if status != L.RMD_OK:
            raise ValueError("invalid DCD header fields")
        return out.tobytes()

    def finish(self, created: str | None = None) -> bytes:
        """The complete file: the header, built last from the real frame count, then the frames."""
        return self.header(created) + b"".join(self.chunks)


def writeRestart(simulation, index: int = 0, velocities: bool = True, box: bool = True,
                 time: float | None = None, title: str = "RainMD restart") -> str:
    """rst7.js:63-101 from the device state. ``time`` defaults to step x timestep when the
    simulation knows both, else 0."""
    if time is None:
        time = float(getattr(simulation, "step", 0)) * float(getattr(simulation, "timestep", 0.0))
    lib = simulation._lib
    size = C.c_int64(0)
    simulation._check(lib.rmd_restart_at(simulation._h, index, title.encode(), float(time),
                                         1 if velocities else 0, 1 if box else 0, None, 0, C.byref(size)))
    buf = C.create_string_buffer(size.value)
    simulation._check(lib.rmd_restart_at(simulation._h, index, title.encode(), float(time),
                                         1 if velocities else 0, 1 if box else 0, buf, size.value,
                                         C.byref(size)))
    return buf.raw[:size.value].decode("ascii")
