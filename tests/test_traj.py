"""On-device trajectory output against the oracle: the DCD frames, the whole DCD file, the
AMBER restart text and the molecule imaging are byte-identical to the reference writers'
(shared/traj/dcd.js, rst7.js, imaging.js as restated in oracle/traj.py) for the same
coordinates and box, and the writers refuse what the reference refuses.
"""
import numpy as np
import pytest

from goldens import system_for
from oracle import traj as ot
from rainmd_b200 import traj
from rainmd_b200.amber import parse_inpcrd
from rainmd_b200.simulation import BatchSimulation, GpuSimulation, NonFiniteStateError

pytestmark = pytest.mark.gpu

ALPHA = 2.6282608939112584


def drifted(system, positions):
    """Three molecules moved by whole lattice vectors (2a - b + 3c), as diffusion leaves them
    (interface.test.js:456-462), so imaging has work to do."""
    a, b, c = np.asarray(system["boxVectors"], np.float64).reshape(3, 3)
    mol = np.asarray(system["topology"]["moleculeOfAtom"])
    p = np.asarray(positions, np.float64).reshape(-1, 3).copy()
    p[np.isin(mol, [1, 2, 3])] += 2 * a - b + 3 * c
    return p.reshape(-1)


def simulation_at(name, run_steps=0, push=True, **options):
    s, pos, _ = system_for(name)
    opts = {"alpha": ALPHA, "grid": [24, 24, 24], "temperature": 300, "seed": 3, "skin": 0.1}
    opts.update(options)
    sim = GpuSimulation(s, opts)
    sim.setState(drifted(s, pos) if push else pos)
    sim.initialise()
    if run_steps:
        sim.minimise(maxIterations=50)
        sim.run(run_steps, blockSize=50)
    return sim, s


def oracle_frame(sim, system, periodic, image, index=0):
    state = sim.readState(index)
    t = system["topology"]
    return ot.dcd_frame(state["positions"].astype(np.float64), state["boxVectors"],
                        t["moleculeOfAtom"], t["moleculeCount"], periodic=periodic, image=image)


@pytest.mark.parametrize("name", ["ala-wat", "ala-oct"])
@pytest.mark.parametrize("periodic,image", [(True, True), (True, False), (False, True), (False, False)])
def test_dcd_frames_are_byte_identical(name, periodic, image):
    sim, s = simulation_at(name, run_steps=100)
    w = traj.DcdWriter(s["topology"]["atomCount"], 0.002, 10, periodic=periodic, molecules=image)
    w.appendFrame(sim)
    assert w.chunks[0] == oracle_frame(sim, s, periodic, image)


def test_dcd_file_is_byte_identical():
    sim, s = simulation_at("ala-wat")
    t = s["topology"]
    w = traj.DcdWriter(t["atomCount"], 0.002, 25, periodic=True, title="RainMD ala-wat")
    expected = []
    for _ in range(3):
        w.appendFrame(sim)
        expected.append(oracle_frame(sim, s, True, True))
        sim.run(25, blockSize=25)
    created = "Created 2026-01-01T00:00:00.000Z"
    head = ot.dcd_header(t["atomCount"], 3, 0, 25, 0.002, True, "RainMD ala-wat", created)
    assert w.finish(created) == head + b"".join(expected)


def test_imaging_is_bitwise_the_oracle():
    sim, s = simulation_at("ala-wat", run_steps=50)
    state = sim.readState()
    t = s["topology"]
    expected = ot.image_molecules(state["positions"].astype(np.float64), state["boxVectors"],
                                  t["moleculeOfAtom"], t["moleculeCount"])
    assert np.array_equal(traj.imageMolecules(sim), expected)


@pytest.mark.parametrize("name", ["ala-wat", "ala-oct"])
def test_restart_text_is_byte_identical_and_round_trips(name):
    sim, s = simulation_at(name, run_steps=100, push=False)
    state = sim.readState()
    text = traj.writeRestart(sim, time=0.2, title=f"RainMD {name}")
    expected = ot.restart_text(state["positions"].astype(np.float64), state["velocities"].astype(np.float64),
                               ot.box_from_vectors(state["boxVectors"]), time=0.2, title=f"RainMD {name}")
    assert text == expected
    again = parse_inpcrd(text, expected_atom_count=s["topology"]["atomCount"])
    assert again["time"] == 0.2
    assert np.max(np.abs(again["positions"] - state["positions"])) < 1e-7
    assert np.max(np.abs(again["velocities"] - state["velocities"])) < 1e-6
    assert traj.writeRestart(sim, velocities=False, box=False, time=0.0) == ot.restart_text(
        state["positions"].astype(np.float64), time=0.0)


def test_batch_writes_each_system_from_its_own_atoms():
    a, pa, _ = system_for("ala-wat")
    b, pb, _ = system_for("ala-wat", cutoff=0.9)
    batch = BatchSimulation([a, b], {"alpha": ALPHA, "grid": [24, 24, 24]})
    batch.setState(0, pa)
    batch.setState(1, drifted(b, pb))
    batch.initialise()
    for k, s in ((0, a), (1, b)):
        w = traj.DcdWriter(s["topology"]["atomCount"], 0.002, 1, periodic=True)
        w.appendFrame(batch, k)
        state = batch.readState(k)
        t = s["topology"]
        assert w.chunks[0] == ot.dcd_frame(state["positions"].astype(np.float64), state["boxVectors"],
                                           t["moleculeOfAtom"], t["moleculeCount"])
        assert traj.writeRestart(batch, k, time=0.0) == ot.restart_text(
            state["positions"].astype(np.float64), state["velocities"].astype(np.float64),
            ot.box_from_vectors(state["boxVectors"]), time=0.0)


def test_writers_refuse_non_finite_and_overwide_coordinates():
    """dcd.js:112-128, rst7.js:27-55: a NaN refuses the frame and the restart; a coordinate
    beyond the 12 columns refuses the restart; the frames before stay."""
    s, pos, _ = system_for("ala-wat")
    sim = GpuSimulation(s, {"alpha": ALPHA, "grid": [24, 24, 24]})
    sim.setState(pos)
    w = traj.DcdWriter(s["topology"]["atomCount"], 0.002, 1, periodic=True)
    w.appendFrame(sim)
    bad = np.asarray(pos, np.float64).copy()
    bad[4] = np.nan
    sim.setState(bad)
    with pytest.raises(NonFiniteStateError, match="DCD writer"):
        w.appendFrame(sim)
    assert w.frameCount == 1
    with pytest.raises(NonFiniteStateError, match="restart writer"):
        traj.writeRestart(sim)
    wide = np.asarray(pos, np.float64).copy()
    wide[0] = 1.0e4  # 100000 angstroms
    sim.setState(wide)
    with pytest.raises(ValueError, match="12-column"):
        traj.writeRestart(sim)
    w.appendFrame(sim)  # a DCD frame has no width limit
    assert w.frameCount == 2
