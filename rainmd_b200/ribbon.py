"""Cartoon ribbon guides, one frame per residue, for the renderer's sweep
(shared/analysis/ribbon.js:110-231).

The host does the sequential half: each residue's side vector is made continuous with the
previous one (flipped when they disagree, so a strand does not corkscrew), strands end in an
arrowhead width profile, and segments (four Catmull-Rom control guides each) never span a
chain break or a hidden residue. The trace (alpha-carbon atom of each residue), the secondary
structure per residue and the chain breaks are inputs, as the reference's `secondary` object
supplies them (shared/analysis/secondary.js).
"""
from __future__ import annotations

import math

import numpy as np

HELIX, SHEET, COIL = "helix", "sheet", "coil"
CROSS_SECTION = {HELIX: (0.120, 0.030), SHEET: (0.110, 0.028), COIL: (0.040, 0.040)}  # half width, half thickness
ARROW_WIDTH = 1.9
ARROW_TIP = 0.012
GUIDE_FLOATS = 12
STRUCTURE_COLOURS = {HELIX: (0.85, 0.37, 0.34), SHEET: (0.92, 0.80, 0.30), COIL: (0.62, 0.64, 0.68)}


def _sub(a, b):
    return [a[0] - b[0], a[1] - b[1], a[2] - b[2]]


def _cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def _dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def _scale(a, k):
    return [a[0] * k, a[1] * k, a[2] * k]


def _normalise(v):
    length = math.sqrt(_dot(v, v))
    return _scale(v, 1 / length) if length > 1e-9 else None


def _any_perpendicular(v):
    axis = [1, 0, 0] if abs(v[0]) < 0.9 else [0, 1, 0]
    return _normalise(_cross(v, axis))


def _runs(length, breaks):
    starts = set(breaks)
    runs, start = [], 0
    for index in range(1, length + 1):
        if index == length or index in starts:
            if index - start >= 2:
                runs.append((start, index))
            start = index
    return runs


def buildRibbon(positions, trace, kinds, breaks=(), visible=None) -> dict:
    """Guides (float32, 12 per kept residue) and segments (uint32, 4 guide indices each)."""
    p = np.asarray(positions, np.float64).reshape(-1)
    kept_trace, kept_kinds, kept_breaks = [], [], []
    brk = set(int(b) for b in breaks)
    previous_kept = -1
    for index, atom in enumerate(trace):
        if visible is not None and not visible[atom]:
            continue
        broke = len(kept_trace) > 0 and (index in brk or previous_kept != index - 1)
        if broke:
            kept_breaks.append(len(kept_trace))
        kept_trace.append(int(atom))
        kept_kinds.append(kinds[index])
        previous_kept = index
    runs = _runs(len(kept_trace), kept_breaks)
    guides = np.zeros(len(kept_trace) * GUIDE_FLOATS, np.float32)
    segments = []
    for start, end in runs:
        def point(offset):
            i = min(max(offset, start), end - 1)
            a = kept_trace[i]
            return [float(p[3 * a]), float(p[3 * a + 1]), float(p[3 * a + 2])]

        previous_side = None
        for index in range(start, end):
            here, before, after = point(index), point(index - 1), point(index + 1)
            tangent = _normalise(_sub(after, before)) or _normalise(_sub(after, here)) or [0, 0, 1]
            midpoint = _scale([before[0] + after[0], before[1] + after[1], before[2] + after[2]], 0.5)
            radial = _sub(here, midpoint)
            radial = _sub(radial, _scale(tangent, _dot(radial, tangent)))
            side = _normalise(_cross(tangent, radial))
            if side is None:
                side = (_any_perpendicular(tangent) if previous_side is None else
                        _normalise(_sub(previous_side, _scale(tangent, _dot(previous_side, tangent))))
                        or _any_perpendicular(tangent))
            if previous_side is not None and _dot(side, previous_side) < 0:
                side = _scale(side, -1)
            previous_side = side
            kind = kept_kinds[index] if kept_kinds[index] in CROSS_SECTION else COIL
            half_width, half_thickness = CROSS_SECTION[kind]
            following = kept_kinds[index + 1] if index + 1 < len(kept_kinds) else None
            after_that = kept_kinds[index + 2] if index + 2 < len(kept_kinds) else None
            if kind == SHEET and following != SHEET:
                half_width = ARROW_TIP
            elif kind == SHEET and following == SHEET and after_that != SHEET:
                half_width *= ARROW_WIDTH
            colour = STRUCTURE_COLOURS.get(kind, STRUCTURE_COLOURS[COIL])
            base = index * GUIDE_FLOATS
            guides[base:base + 12] = [*here, half_width, *side, half_thickness, *colour, 0]
        for index in range(start, end - 1):
            segments += [max(index - 1, start), index, index + 1, min(index + 2, end - 1)]
    return {"guides": guides, "segments": np.asarray(segments, np.uint32), "segmentCount": len(segments) // 4,
            "guideCount": len(kept_trace), "runCount": len(runs)}
