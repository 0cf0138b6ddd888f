"""The CUDA renderer against its CPU restatement (oracle/raster.c): the viewer's sphere
impostors and cartoon ribbon (web/viewer.js:83-308) drawn into the same RGBA8 image, bit for
bit, from several camera positions, with hidden atoms, from a simulation's device positions and
from host coordinates."""
import numpy as np
import pytest

import oracle
import traces
from goldens import system_for
from rainmd_b200.ribbon import buildRibbon
from rainmd_b200.simulation import BatchSimulation, GpuSimulation
from rainmd_b200.viewer import StructureViewer

pytestmark = pytest.mark.gpu

ALPHA = 2.6282608939112584


def oracle_image(viewer, positions, ribbon=None):
    spheres = viewer.representation != "ribbon"
    rb = ribbon if viewer.representation != "spheres" else None
    return oracle.render(np.asarray(positions, np.float32).reshape(-1), viewer.camera(), viewer.styles,
                         None if rb is None else rb["guides"], None if rb is None else rb["segments"],
                         spheres=spheres, ribbon=rb is not None, width=viewer.width, height=viewer.height)


def protein_ribbon(offset):
    positions, kinds = traces.mixed()
    positions = positions + offset
    return buildRibbon(positions.reshape(-1), list(range(len(positions))), kinds)


@pytest.mark.parametrize("azimuth,elevation,scale", [(0.6, 0.35, 1.0), (2.2, -0.8, 0.7), (-1.0, 1.2, 0.25)])
def test_spheres_match_the_oracle(azimuth, elevation, scale):
    s, pos, _ = system_for("ala-wat")
    sim = GpuSimulation(s, {"alpha": ALPHA, "grid": [24, 24, 24]})
    sim.setState(pos)
    v = StructureViewer(96, 72)
    v.setStructure(s["topology"], positions=pos)
    v.azimuth, v.elevation, v.distance = azimuth, elevation, v.distance * scale
    image = v.draw(sim)
    state = sim.readState()
    expected = oracle_image(v, state["positions"])
    assert image.shape == (72, 96, 4)
    assert np.array_equal(image, expected)
    assert (image[..., :3] != expected[0, 0, :3]).any()  # something was drawn


def test_ribbon_and_spheres_together_match_the_oracle():
    ribbon = protein_ribbon(np.array([0.5, 0.5, 0.5]))
    positions, _ = traces.mixed()
    topology = {"atomCount": len(positions), "atomicNumbers": [6] * len(positions)}
    v = StructureViewer(128, 96)
    v.setStructure(topology, positions=positions + 0.5, radiusScale=0.4)
    v.setRibbon(ribbon)
    for mode in ("ribbon", "both"):
        v.representation = mode
        for az in (0.3, 1.9, 4.0):
            v.azimuth = az
            image = v.draw(positions=positions + 0.5)
            assert np.array_equal(image, oracle_image(v, positions + 0.5, ribbon)), (mode, az)


def test_hidden_atoms_and_host_coordinates():
    s, pos, _ = system_for("ala-wat")
    t = s["topology"]
    sim = GpuSimulation(s, {"alpha": ALPHA, "grid": [24, 24, 24]})
    sim.setState(pos)
    visible = np.zeros(t["atomCount"], np.uint8)
    visible[:22] = 1  # the solute only
    v = StructureViewer(80, 60)
    v.setStructure(t, visible=visible, heavyOnly=True, positions=pos)
    from_device = v.draw(sim)
    from_host = v.draw(positions=sim.readState()["positions"])
    assert np.array_equal(from_device, from_host)
    assert np.array_equal(from_device, oracle_image(v, sim.readState()["positions"]))


def test_batch_renders_its_own_system():
    a, pa, _ = system_for("ala-wat")
    b, pb, _ = system_for("ala-wat", cutoff=0.9)
    batch = BatchSimulation([a, b], {"alpha": ALPHA, "grid": [24, 24, 24]})
    batch.setState(0, pa)
    batch.setState(1, np.asarray(pb).reshape(-1) + 0.3)
    v = StructureViewer(64, 48)
    v.setStructure(b["topology"], positions=np.asarray(pb).reshape(-1) + 0.3)
    image = v.draw(batch, 1)
    assert np.array_equal(image, oracle_image(v, batch.readState(1)["positions"]))
