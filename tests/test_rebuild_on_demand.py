"""Neighbour lists rebuilt on demand: each step the device compares the largest displacement
since the last build with half the skin and runs the rebuild (an IF node of the step graph)
exactly when a pair could have come within the cutoff unseen. The reference rebuilds on a
host schedule adapted between blocks (simulation.js:544-623), which it checks after the fact;
here no force evaluation uses a stale list, and every build inside a block still reports its
neighbour requirement to the capacity check (cells.js:282-288).
"""
import numpy as np
import pytest

from goldens import system_for
from rainmd_b200.simulation import GpuSimulation

pytestmark = pytest.mark.gpu

ALPHA = 2.6282608939112584


def make(**options):
    s, pos, _ = system_for("ala-wat")
    opts = {"alpha": ALPHA, "grid": [24, 24, 24], "temperature": 300, "seed": 11, "dispersionCorrection": False}
    opts.update(options)
    sim = GpuSimulation(s, opts)
    sim.setState(pos)
    sim.initialise()
    sim.minimise(maxIterations=50)
    return sim


@pytest.mark.parametrize("skin", [0.04, 0.1])
def test_lists_in_hand_are_never_stale(skin):
    """After 300 steps in blocks of 100, the forces of the last step (computed with the list
    the device kept) equal the forces from a list built afresh at the same positions."""
    sim = make(skin=skin)
    before = sim.diagnostics()["list_builds"]
    sim.run(300, blockSize=100)
    d = sim.diagnostics()
    assert d["rebuild_on_demand"] == 1
    builds = d["list_builds"] - before
    assert 0 < builds < 300
    assert d["skin_violations"] == 0 and d["worst_skin_usage"] <= 1.0
    kept = sim.readState()["forces"].astype(np.float64)
    _, fresh = sim.debugEvaluate()
    rms = np.sqrt(np.mean(fresh ** 2))
    assert np.max(np.abs(kept - fresh)) < 1e-5 * rms


def test_a_thinner_skin_rebuilds_more_often():
    counts = []
    for skin in (0.04, 0.15):
        sim = make(skin=skin)
        before = sim.diagnostics()["list_builds"]
        sim.run(200, blockSize=100)
        counts.append(sim.diagnostics()["list_builds"] - before)
        sim.release()
    assert counts[0] > counts[1] >= 1


def test_reference_schedule_is_kept_when_asked():
    """rebuildOnDemand = False: the reference's fixed interval. The minimiser leaves a fresh
    list, so 100 steps build at steps 5, 10, ..., 95."""
    sim = make(rebuildOnDemand=False, rebuildInterval=5, adaptiveRebuild=False, skin=0.15)
    before = sim.diagnostics()["list_builds"]
    sim.run(100, blockSize=50)
    d = sim.diagnostics()
    assert d["rebuild_on_demand"] == 0
    assert d["list_builds"] - before == 19


def test_requirement_of_every_build_in_a_block_is_checked():
    """A list sized to exactly what the starting structure needs, then 400 steps in one
    block: if any build inside the block needed more room than the list had, the block check
    sees it and grows the list (it would otherwise see only the block's last build)."""
    probe = make(skin=0.08)
    state = probe.readState()
    need = probe.diagnostics()["neighbour_required"]
    probe.release()
    s, _, _ = system_for("ala-wat")
    sim = GpuSimulation(s, {"alpha": ALPHA, "grid": [24, 24, 24], "temperature": 300, "seed": 11,
                            "dispersionCorrection": False, "skin": 0.08, "maxNeighbours": need})
    sim.setState(state["positions"].astype(np.float64), state["velocities"].astype(np.float64))
    sim.initialise()
    d0 = sim.diagnostics()
    assert d0["neighbour_growths"] == 0
    sim.run(400, blockSize=400)
    d = sim.diagnostics()
    if d["worst_neighbour_required"] > d0["neighbour_capacity"]:
        assert d["neighbour_growths"] >= 1 and d["neighbour_capacity"] >= d["worst_neighbour_required"]
    else:
        assert d["neighbour_growths"] == 0


def test_batch_rebuilds_only_stale_systems_and_none_is_stale():
    """Three systems in one handle, with thin and thick skins: each system's lists are
    rebuilt when that system needs it, and after 300 steps every system's last forces equal
    the forces from lists built afresh."""
    from rainmd_b200 import synthetic
    from rainmd_b200.simulation import BatchSimulation
    from rainmd_b200.topology import build_system

    made = synthetic.batch(3, low=1000, high=2500, seed=9)
    built = [build_system(t, cutoff=0.9) for t, _ in made]
    batch = BatchSimulation(built, {"pmeOrder": 4, "skin": 0.06, "temperature": 300, "seed": 2})
    for k, (_, pos) in enumerate(made):
        batch.setState(k, pos)
    batch.initialise()
    batch.minimise(maxIterations=50)
    before = batch.diagnostics()["list_builds"]
    batch.run(300, blockSize=100)
    assert batch.diagnostics()["list_builds"] > before
    kept = [batch.readState(k)["forces"].astype(np.float64) for k in range(3)]
    for k in range(3):
        _, fresh = batch.debugEvaluate(k)
        rms = np.sqrt(np.mean(fresh ** 2))
        assert np.max(np.abs(kept[k] - fresh)) < 1e-5 * rms, k
