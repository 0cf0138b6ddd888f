"""The viewer's host half: ribbon guides (shared/analysis/ribbon.js:110-231, with the
reference's ribbon tests, test/interface.test.js:537-676, restated on synthetic traces), the
camera uniform and the styles (web/viewer.js:418-510, 632-692); and the renderer's refusal of
segments that name guides which do not exist (no GPU needed)."""
import ctypes as C
import math

import numpy as np
import pytest

import traces
from goldens import system_for
from rainmd_b200 import _lib as L
from rainmd_b200.ribbon import GUIDE_FLOATS, buildRibbon
from rainmd_b200.viewer import RmdCamera, StructureViewer


def build(positions, kinds, breaks=(), visible=None):
    n = len(positions)
    return buildRibbon(np.asarray(positions).reshape(-1), list(range(n)), kinds, breaks, visible)


def field(ribbon, index, offset):
    return ribbon["guides"][index * GUIDE_FLOATS + offset: index * GUIDE_FLOATS + offset + 3].astype(np.float64)


CASES = {
    "helix": lambda: build(traces.helix(), ["helix"] * 24),
    "strand": lambda: build(traces.strand(), ["sheet"] * 24),
    "mixed": lambda: build(*traces.mixed()),
}


@pytest.mark.parametrize("name", list(CASES))
def test_frames_are_unit_perpendicular_and_never_flip(name):
    ribbon = CASES[name]()
    assert ribbon["segmentCount"] == ribbon["guideCount"] - 1
    worst = 1.0
    for index in range(1, ribbon["guideCount"] - 1):
        side = field(ribbon, index, 4)
        assert abs(np.linalg.norm(side) - 1) < 1e-5
        tangent = field(ribbon, index + 1, 0) - field(ribbon, index - 1, 0)
        assert abs(side @ tangent / np.linalg.norm(tangent)) < 1e-5
    for index in range(1, ribbon["guideCount"]):
        worst = min(worst, field(ribbon, index, 4) @ field(ribbon, index - 1, 4))
    assert worst > 0


def test_strand_arrowhead_and_constant_helix():
    strand = CASES["strand"]()
    widths = strand["guides"][3::GUIDE_FLOATS]
    assert widths[-2] > widths[0] * 1.5 and 0 < widths[-1] < widths[0] * 0.25
    helix = CASES["helix"]()
    assert len(set(np.round(helix["guides"][3::GUIDE_FLOATS], 4))) == 1
    positions, kinds = traces.mixed()
    mixed = build(positions, kinds)
    w = mixed["guides"][3::GUIDE_FLOATS]
    assert w[kinds.index("coil")] < 0.5 * w[kinds.index("helix")]


def test_breaks_and_hidden_residues_split_runs():
    positions, kinds = traces.mixed()
    whole = build(positions, kinds)
    assert whole["runCount"] == 1
    visible = np.ones(len(positions), np.uint8)
    visible[len(positions) // 2] = 0
    split = build(positions, kinds, visible=visible)
    assert split["guideCount"] == whole["guideCount"] - 1 and split["runCount"] == 2
    assert split["segmentCount"] == whole["segmentCount"] - 2
    two = build(positions, kinds, breaks=[10])
    assert two["runCount"] == 2 and two["segmentCount"] == two["guideCount"] - 2
    for ribbon in (whole, split, two):
        seg = ribbon["segments"].reshape(-1, 4)
        assert np.all(seg < ribbon["guideCount"])
        assert np.all(seg[:, 2] - seg[:, 1] == 1)
        assert np.all(seg[:, 0] <= seg[:, 1]) and np.all(seg[:, 3] >= seg[:, 2])


def test_camera_uniform_is_the_viewer_draw_uniform():
    v = StructureViewer(640, 480)
    u = v.camera()
    assert u.dtype == np.float32 and u.shape == (36,)
    right, up, forward = u[16:19].astype(float), u[20:23].astype(float), u[24:27].astype(float)
    for a in (right, up, forward):
        assert abs(np.linalg.norm(a) - 1) < 1e-6
    assert abs(right @ up) < 1e-6 and abs(right @ forward) < 1e-6 and abs(up @ forward) < 1e-6
    # the eye is `distance` along forward from the centre: it projects to w = 0 (clip w = -z_view)
    vp = u[:16].reshape(4, 4).T.astype(float)
    eye = forward * v.distance
    clip = vp @ np.append(eye, 1.0)
    assert abs(clip[3]) < 1e-4
    centre = vp @ np.array([0.0, 0.0, 0.0, 1.0])
    assert abs(centre[0] / centre[3]) < 1e-6 and abs(centre[1] / centre[3]) < 1e-6


def test_styles_and_framing():
    s, pos, _ = system_for("ala-wat")
    t = s["topology"]
    v = StructureViewer(64, 48)
    v.setStructure(t, heavyOnly=True, positions=pos)
    radius = v.styles[:, 3]
    numbers = np.asarray(t["atomicNumbers"])
    assert np.all(radius[numbers == 1] == 0)
    assert np.allclose(radius[numbers == 8], np.float32(0.152 * 0.65))
    assert v.distance > 0 and len(v.centre) == 3


def test_renderer_refuses_segments_naming_missing_guides():
    lib = L.load()
    cam = RmdCamera.from_buffer_copy(StructureViewer(8, 8).camera().tobytes())
    guides = np.zeros(12 * 3, np.float32)
    segments = np.array([0, 1, 2, 3], np.uint32)  # guide 3 of 3
    out = np.zeros(8 * 8 * 4, np.uint8)
    fp = C.POINTER(C.c_float)
    status = lib.rmd_render_positions(None, 0, C.byref(cam), None, guides.ctypes.data_as(fp), 3,
                                      segments.ctypes.data_as(C.POINTER(C.c_uint32)), 1, 0, 1, 8, 8,
                                      out.ctypes.data_as(C.POINTER(C.c_uint8)))
    assert status == L.RMD_ERR_INVALID
    assert b"names guide 3 of 3" in lib.rmd_last_error(None)
