"""Headless structure viewer: the reference's StructureViewer (web/viewer.js:330-724) with its
canvas replaced by an RGBA8 image that CUDA draws (rainmd_b200/csrc/raster.cu).

The host half is the reference's host half: per-atom styles from the element table and the
visibility options (viewer.js:440-470), framing (viewer.js:485-510), and the camera uniform
each draw() builds in float64 and rounds to float32 (viewer.js:632-692). The two render passes,
sphere impostors and the cartoon ribbon, run on the device from the simulation's own position
buffer (or from host coordinates when there is no simulation yet), and the image comes back as
an array [height, width, 4].
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib as L

# CPK-ish colours and van der Waals radii (nm) by atomic number (viewer.js:30-41)
ELEMENTS = {
    1: ((0.95, 0.95, 0.95), 0.110), 6: ((0.35, 0.37, 0.40), 0.170), 7: ((0.22, 0.38, 0.85), 0.155),
    8: ((0.88, 0.25, 0.20), 0.152), 11: ((0.55, 0.35, 0.85), 0.227), 12: ((0.20, 0.70, 0.30), 0.173),
    15: ((0.95, 0.60, 0.15), 0.180), 16: ((0.92, 0.85, 0.25), 0.180), 17: ((0.25, 0.80, 0.35), 0.175),
}
DEFAULT_ELEMENT = ((0.75, 0.45, 0.85), 0.160)


class RmdCamera(C.Structure):
    _fields_ = [("view_projection", C.c_float * 16), ("right", C.c_float * 4), ("up", C.c_float * 4),
                ("forward", C.c_float * 4), ("centre", C.c_float * 4)]


def _script_hypot(*values):
    """Math.hypot: scaled by the largest magnitude, Kahan-compensated sum of squares."""
    v = [abs(float(x)) for x in values]
    top = max(v)
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


def _perspective(fov, aspect, near, far):
    f = 1 / math.tan(fov / 2)
    rng = 1 / (near - far)
    return [f / aspect, 0, 0, 0, 0, f, 0, 0, 0, 0, far * rng, -1, 0, 0, near * far * rng, 0]


def _multiply(a, b):
    """viewer.js:317-327: float64 sums of a (numbers) times b (float32), rounded to float32."""
    out = np.zeros(16, np.float32)
    for column in range(4):
        for row in range(4):
            total = 0.0
            for k in range(4):
                total += a[k * 4 + row] * float(b[column * 4 + k])
            out[column * 4 + row] = total
    return out


class StructureViewer:
    def __init__(self, width: int = 800, height: int = 600):
        self.width, self.height = int(width), int(height)
        self.azimuth = 0.6
        self.elevation = 0.35
        self.distance = 6.0
        self.centre = [0.0, 0.0, 0.0]
        self.atomCount = 0
        self.styles = None
        self.representation = "spheres"  # "spheres", "ribbon" or "both"
        self.ribbon = None
        self._lib = L.load()

    def setStructure(self, topology: dict, visible=None, heavyOnly: bool = False, radiusScale: float = 0.65,
                     colours=None, positions=None, box=None):
        """Per-atom colour and radius (viewer.js:418-470): element colours unless `colours`
        ([N, 3]) is given; a hidden atom (not `visible`, or a hydrogen under `heavyOnly`) has
        radius 0."""
        n = int(topology["atomCount"])
        self.atomCount = n
        numbers = topology.get("atomicNumbers")
        styles = np.zeros((n, 4), np.float32)
        for atom in range(n):
            z = int(numbers[atom]) if numbers is not None else 0
            colour, radius = ELEMENTS.get(z, DEFAULT_ELEMENT)
            if colours is not None:
                colour = colours[atom]
            hidden = (visible is not None and not visible[atom]) or (heavyOnly and z == 1)
            styles[atom, :3] = colour
            styles[atom, 3] = 0.0 if hidden else radius * radiusScale
        self.styles = styles
        if positions is not None:
            self.frame(positions, styles)
        elif box is not None:
            self.centre = [length / 2 for length in box["lengths"]]
            self.distance = max(box["lengths"]) * 1.9

    def frame(self, positions, styles=None):
        """Point the camera at the visible atoms (viewer.js:485-510)."""
        styles = self.styles if styles is None else styles
        p = np.asarray(positions, np.float64).reshape(-1, 3)
        shown = np.asarray(styles)[:, 3] > 0
        if not shown.any():
            return
        low, high = p[shown].min(0), p[shown].max(0)
        self.centre = [(float(low[k]) + float(high[k])) / 2 for k in range(3)]
        extent = max(float(high[0] - low[0]), float(high[1] - low[1]), float(high[2] - low[2]), 0.5)
        self.distance = (0.5 * extent * 1.45) / math.tan(0.45)

    def setRibbon(self, ribbon: dict | None):
        """A ribbon as buildRibbon returns it (rainmd_b200/ribbon.py)."""
        self.ribbon = ribbon

    def camera(self) -> np.ndarray:
        """The 36-float uniform draw() writes (viewer.js:651-692)."""
        ce = math.cos(self.elevation)
        eye = [self.distance * ce * math.sin(self.azimuth), self.distance * math.sin(self.elevation),
               self.distance * ce * math.cos(self.azimuth)]
        forward = [v / self.distance for v in eye]
        up0 = [0, 1, 0]
        right = [up0[1] * forward[2] - up0[2] * forward[1], up0[2] * forward[0] - up0[0] * forward[2],
                 up0[0] * forward[1] - up0[1] * forward[0]]
        length = _script_hypot(*right) or 1
        right = [v / length for v in right]
        up = [forward[1] * right[2] - forward[2] * right[1], forward[2] * right[0] - forward[0] * right[2],
              forward[0] * right[1] - forward[1] * right[0]]
        view = np.array([
            right[0], up[0], forward[0], 0, right[1], up[1], forward[1], 0, right[2], up[2], forward[2], 0,
            -(right[0] * eye[0] + right[1] * eye[1] + right[2] * eye[2]),
            -(up[0] * eye[0] + up[1] * eye[1] + up[2] * eye[2]),
            -(forward[0] * eye[0] + forward[1] * eye[1] + forward[2] * eye[2]), 1], np.float32)
        projection = _perspective(0.9, self.width / self.height, 0.05, self.distance * 6 + 20)
        uniform = np.zeros(36, np.float32)
        uniform[:16] = _multiply(projection, view)
        uniform[16:19] = right
        uniform[20:23] = up
        uniform[24:27] = forward
        uniform[28:31] = self.centre
        return uniform

    def draw(self, simulation=None, index: int = 0, positions=None) -> np.ndarray:
        """Render the current structure: from `simulation`'s device positions, or from host
        `positions` (StructureViewer.upload). Returns RGBA8 [height, width, 4], row 0 on top."""
        if self.styles is None:
            raise ValueError("setStructure first")
        cam = RmdCamera.from_buffer_copy(self.camera().tobytes())
        spheres = self.representation != "ribbon"
        rb = self.ribbon if self.representation != "spheres" else None
        guides = segments = None
        guide_count = segment_count = 0
        if rb is not None and rb["segmentCount"] > 0:
            guides = np.ascontiguousarray(rb["guides"], np.float32)
            segments = np.ascontiguousarray(rb["segments"], np.uint32)
            guide_count, segment_count = len(guides) // 12, len(segments) // 4
        out = np.zeros((self.height, self.width, 4), np.uint8)
        fp = C.POINTER(C.c_float)
        styles = np.ascontiguousarray(self.styles, np.float32)
        g = guides.ctypes.data_as(fp) if guides is not None else None
        s = segments.ctypes.data_as(C.POINTER(C.c_uint32)) if segments is not None else None
        args = (C.byref(cam), styles.ctypes.data_as(fp), g, guide_count, s, segment_count,
                1 if spheres else 0, 1 if segment_count else 0, self.width, self.height,
                out.ctypes.data_as(C.POINTER(C.c_uint8)))
        if simulation is not None:
            simulation._check(self._lib.rmd_render_at(simulation._h, index, *args))
        else:
            p = np.ascontiguousarray(positions, np.float32).reshape(-1)
            status = self._lib.rmd_render_positions(p.ctypes.data_as(fp), len(p) // 3, *args)
            if status != L.RMD_OK:
                raise ValueError(self._lib.rmd_last_error(None).decode())
        return out
