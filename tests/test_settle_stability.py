"""SETTLE's long-run energy conservation: constant-energy dynamics (no thermostat) of a
23,558-atom water box keeps its total energy and temperature. A SETTLE formed from absolute
f32 coordinates heats such a box exponentially (its temperature doubles every ~5 ps); this
is the guard against that."""
import numpy as np
import pytest

from rainmd_b200 import synthetic
from rainmd_b200.simulation import GpuSimulation
from rainmd_b200.topology import build_system

pytestmark = pytest.mark.gpu


def test_settle_conserves_energy_without_a_thermostat():
    topo, pos = synthetic.water_box(23558, seed=3)
    system = build_system(topo, cutoff=0.9)
    options = {"pmeOrder": 4, "grid": [64, 64, 64], "waterSolver": 1, "skin": 0.15, "rebuildInterval": 10,
               "temperature": 300.0, "seed": 3, "dispersionCorrection": True}
    sim = GpuSimulation(system, options)
    sim.setState(pos)
    sim.initialise()
    sim.minimise(maxIterations=200, forceTolerance=1000.0)
    sim.run(3000, blockSize=100)
    state = sim.readState()
    nve = GpuSimulation(system, dict(options, friction=0.0))
    nve.setState(state["positions"].astype(np.float64), state["velocities"].astype(np.float64))
    nve.initialise()
    first = nve.energy()
    nve.run(10000, blockSize=100)  # 20 ps
    last = nve.energy()
    drift_per_atom = abs(last["total"] - first["total"]) / system["topology"]["atomCount"]
    assert drift_per_atom < 0.002, (first["total"], last["total"])
    assert 270.0 < last["temperature"] < 330.0
