"""The engine's cell plan against the reference's planning functions, on the host.

rmd_plan_system runs the same host code rmd_create plans each system with (skinFor,
planCellList, pmeParameters) and needs no GPU; the oracle restates shared/topology/cells.js
in Python floats. The skin, cell counts, stencil, neighbour estimate and capacity, and the
grown capacity after an overflow, must agree for every geometry the tests and the benchmark
use: the golden fixtures at four cutoffs, the sheared (octahedral) box, the water boxes of the
precision study and the benchmark, and the 1,190-atom chain system.
"""
import math

import pytest

import oracle
from goldens import system_for
from rainmd_b200 import synthetic
from rainmd_b200.simulation import grownCapacity, planSystem
from rainmd_b200.topology import build_system


def _systems():
    out = []
    for cutoff in (0.5, 0.7, 1.0, 1.25):
        s, _, _ = system_for("ala-wat", cutoff=cutoff)
        out.append((f"ala-wat rc {cutoff}", s))
    s, _, _ = system_for("ala-oct")
    out.append(("ala-oct", s))
    for n in (2854, 23558):
        topo, _ = synthetic.water_box(n, seed=1)
        out.append((f"water-{n}", build_system(topo, cutoff=0.9)))
    topo, _ = synthetic.config0(seed=1)
    out.append(("chain-1190", build_system(topo, cutoff=0.9)))
    return out


SYSTEMS = _systems()


def row_capacity(max_neighbours):
    return (max_neighbours + 3) // 4 * 4


@pytest.mark.parametrize("name,system", SYSTEMS, ids=[n for n, _ in SYSTEMS])
@pytest.mark.parametrize("options", [
    {},                                               # skinFor at the defaults (2 fs, 298 K)
    {"timestep": 0.004, "temperature": 350.0},        # skinFor scaled, and capped by the box
    {"skin": 0.15},                                   # the benchmark's skin
    {"skin": 0.1, "neighbourSlack": 1.6},
    {"skin": 0.1, "maxNeighbours": 64},
])
def test_plan_matches_cells_js(name, system, options):
    box = system["boxVectors"]
    cutoff = system["options"]["cutoff"]
    n = system["topology"]["atomCount"]
    plan = planSystem(system, options)
    skin = options.get("skin")
    if skin is None:
        skin = oracle.skin_for(system["topology"]["masses"], box, cutoff,
                               timestep=options.get("timestep", 0.002),
                               temperature=options.get("temperature", 298.0))
    expect = oracle.plan_cell_list(n, box, cutoff, skin=skin,
                                   neighbour_slack=options.get("neighbourSlack", 2.0),
                                   max_neighbours=options.get("maxNeighbours"))
    assert plan["skin"] == skin
    assert plan["list_cutoff"] == expect["listCutoff"]
    assert plan["counts"] == expect["counts"]
    assert plan["cell_count"] == expect["cellCount"]
    assert plan["stencil_cells"] == len(expect["stencil"])
    assert math.isclose(plan["estimated_neighbours"], expect["estimatedNeighbours"], rel_tol=1e-13)
    assert plan["max_neighbours"] == expect["maxNeighbours"]
    assert plan["capacity"] == row_capacity(expect["maxNeighbours"])
    assert math.isclose(plan["mean_occupancy"], expect["meanOccupancy"], rel_tol=1e-15)


@pytest.mark.parametrize("name,system", SYSTEMS, ids=[n for n, _ in SYSTEMS])
def test_pme_parameters_match_parameters_js(name, system):
    """pmeParameters (shared/pme/parameters.js:43-49, 90-100): alpha from the Ewald tolerance
    and the smallest 2/3/5-smooth grid per axis, when neither is given."""
    cutoff = system["options"]["cutoff"]
    plan = planSystem(system, {"ewaldTolerance": 5e-4})
    alpha = oracle.alpha_from_tolerance(cutoff, 5e-4)
    assert plan["alpha"] == pytest.approx(alpha, rel=1e-15)
    assert plan["grid"] == list(oracle.grid_size_for(system["boxVectors"], alpha, 5e-4))


def test_skin_is_capped_by_the_box():
    """skinFor's cap (cells.js:78-84): a hot, long-timestep run in the 2.265 nm box asks for more
    skin than fits between the cutoff and half the box, and gets 0.9 of the room."""
    topo, _ = synthetic.config0(seed=1)
    system = build_system(topo, cutoff=0.9)
    plan = planSystem(system, {"timestep": 0.004, "temperature": 400.0})
    room = min(system["boxVectors"][0], system["boxVectors"][4], system["boxVectors"][8]) / 2 - 0.9
    assert plan["skin"] == pytest.approx(0.9 * room, rel=1e-15)


@pytest.mark.parametrize("capacity", [32, 64, 300, 1020])
@pytest.mark.parametrize("required", [0, 33, 65, 301, 526, 1500])
def test_grown_capacity_matches_grown_plan(capacity, required):
    assert grownCapacity(capacity, required) == row_capacity(oracle.grown_plan(capacity, required))


def test_planned_counts_reach_the_benchmark_geometry():
    """The 23,558-atom benchmark box (6.18 nm, rc 0.9, skin 0.15): 5 cells per axis, the full
    27-cell stencil, and a capacity near twice the ~510 partners within 1.05 nm."""
    topo, _ = synthetic.water_box(23558, seed=1)
    plan = planSystem(build_system(topo, cutoff=0.9), {"skin": 0.15})
    assert plan["counts"] == [5, 5, 5] and plan["stencil_cells"] == 27
    assert 400 < plan["estimated_neighbours"] < 600
    assert plan["capacity"] % 4 == 0 and plan["capacity"] >= 2 * plan["estimated_neighbours"]
