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
    """Per-atom rows (pair_list 1), the form whose search-group size and pair-loop lanes are
    tuned; the group-pair rows have one shape of each."""
    opts = {"pmeOrder": 4, "grid": [32, 32, 32], "skin": 0.1, "temperature": 300.0, "seed": 5, "pairList": 1}
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


def test_group_pair_rows_tune_the_row_split_and_the_spreading():
    """Group-pair rows: 4-atom search groups always; the warps sharing a row (1, 2 or 4: 32, 64
    or 128 lanes a row) and the spreading block are timed and the fastest kept."""
    system, pos = water()
    sim = make(system, pos, pairList=0)
    shapes = sim.kernelShapes()
    assert shapes["neighbourGroupAtoms"] == 4 and shapes["tuned"]["neighbourGroupAtoms"] == {}
    for name, candidates in (("nonbondedLanes", [32, 64, 128]), ("spreadAtomsPerBlock", [4, 8, 16])):
        tuned = shapes["tuned"][name]
        assert sorted(tuned) == candidates, name
        assert shapes[name] == min(tuned, key=tuned.get), name
    sim.release()


def test_group_pair_rows_give_the_per_atom_rows_results_bit_for_bit():
    """Each pair's force is quantised from the same f32 operands whichever structure lists it,
    so both structures sum the same integers: forces, energies, a minimisation and a run agree
    bit for bit, and so does a group-pair run whose builds also write the per-atom rows."""
    system, pos = water()
    results = []
    for form, lanes in ((1, 16), (0, 32), (2, 128), (0, 64)):
        sim = make(system, pos, pairList=form, spreadAtomsPerBlock=8, nonbondedLanes=lanes)
        energy, forces = sim.debugEvaluate()
        sim.minimise(maxIterations=20)
        sim.run(40, blockSize=10)
        e = sim.energy()
        state = sim.readState()
        results.append((energy, forces, e, state))
        sim.release()
    (e1, f1, end1, s1) = results[0]
    for (e2, f2, end2, s2) in results[1:]:
        assert np.array_equal(f1, f2)
        for key in ("lennard_jones", "coulomb_direct", "coulomb_reciprocal", "potential"):
            assert e1[key] == e2[key], key
        for key in ("lennardJones", "coulombDirect", "coulombReciprocal", "potential", "kinetic"):
            assert end1[key] == end2[key], key
        assert np.array_equal(s1["positions"], s2["positions"])
        assert np.array_equal(s1["velocities"], s2["velocities"])
        assert np.array_equal(s1["forces"], s2["forces"])
