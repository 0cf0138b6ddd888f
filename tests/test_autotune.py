"""The kernel-shape autotuner: every shape it may pick gives the same lists, forces and
energies, and when shapes are left to it, it times every candidate and keeps the fastest.
"""
import numpy as np
import pytest

from rainmd_b200 import synthetic
from rainmd_b200.simulation import GpuSimulation
from rainmd_b200.topology import build_system

pytestmark = pytest.mark.gpu


def water(n=2854, seed=3):
    topo, pos = synthetic.water_box(n, seed=seed)
    system = build_system(topo, constraints="HBonds", rigid_water=True, cutoff=0.9)
    return system, pos


def make(system, pos, **shapes):
    opts = {"pmeOrder": 4, "grid": [32, 32, 32], "skin": 0.1, "temperature": 300.0, "seed": 5}
    opts.update(shapes)
    sim = GpuSimulation(system, opts)
    sim.setState(pos)
    sim.initialise()
    return sim


def test_autotuner_times_every_candidate_and_keeps_the_fastest():
    system, pos = water()
    sim = make(system, pos)
    shapes = sim.kernelShapes()
    for name, candidates in (("neighbourGroupAtoms", (4, 8, 16)), ("nonbondedLanes", (8, 16, 32)),
                             ("spreadAtomsPerBlock", (4, 8, 16))):
        tuned = shapes["tuned"][name]
        assert sorted(tuned) == list(candidates), name
        assert all(t > 0 for t in tuned.values())
        assert shapes[name] == min(tuned, key=tuned.get), name


def test_fixed_shapes_are_not_tuned():
    system, pos = water()
    sim = make(system, pos, neighbourGroupAtoms=16, nonbondedLanes=8, spreadAtomsPerBlock=4)
    shapes = sim.kernelShapes()
    assert (shapes["neighbourGroupAtoms"], shapes["nonbondedLanes"], shapes["spreadAtomsPerBlock"]) == (16, 8, 4)
    assert shapes["tuned"] == {"neighbourGroupAtoms": {}, "nonbondedLanes": {}, "spreadAtomsPerBlock": {}}


def test_every_shape_gives_bitwise_identical_results():
    """Fixed-point pair forces and charge grid: the launch shape cannot change a bit."""
    system, pos = water()
    reference = None
    for group, lanes, spread in ((8, 32, 8), (16, 16, 4), (32, 8, 16), (4, 8, 4), (32, 32, 16)):
        sim = make(system, pos, neighbourGroupAtoms=group, nonbondedLanes=lanes, spreadAtomsPerBlock=spread)
        energy, forces = sim.debugEvaluate()
        cap, counts, rows, required = sim.debugNeighbours()
        lists = [rows[i, :counts[i]].copy() for i in range(len(counts))]
        sim.minimise(maxIterations=20)
        sim.run(20, blockSize=10)
        state = sim.readState()
        got = (energy["potential"], forces, lists, state["positions"])
        if reference is None:
            reference = got
            continue
        assert got[0] == reference[0]
        assert np.array_equal(got[1], reference[1])
        assert all(np.array_equal(a, b) for a, b in zip(got[2], reference[2]))
        assert np.array_equal(got[3], reference[3])
        sim.release()
