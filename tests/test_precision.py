"""The precision form against the FP64 oracle on pure TIP3P water boxes of 2,854, 23,558 and
99,999 atoms at 0.997 g/cm^3 (PME order 4 at <= 1 A grid spacing, 0.9 nm cutoff): FP32 pair
and PME arithmetic with every pair force and pair energy quantised to 64-bit fixed point
(2^32 per unit) before summing, FP64 energy reductions. Every energy term within 1e-5
relative of the oracle, evaluated after minimisation and 1,000 steps of MD at the f32
coordinates the device holds."""
import math

import numpy as np
import pytest

import oracle
from rainmd_b200 import synthetic
from rainmd_b200.simulation import GpuSimulation
from rainmd_b200.topology import build_system

pytestmark = pytest.mark.gpu

CUTOFF = 0.9
ALPHA = math.sqrt(-math.log(2.0 * 5e-4)) / CUTOFF  # Ewald tolerance 5e-4 (parameters.js:43-49)


def smooth_at_least(n):
    while True:
        r = n
        for p in (2, 3, 5):
            while r % p == 0:
                r //= p
        if r == 1:
            return n
        n += 1


def precision_case(n_atoms, seed=1):
    topo, pos = synthetic.water_box(n_atoms, seed=seed)
    system = build_system(topo, cutoff=CUTOFF)
    box = system["boxVectors"]
    grid = [smooth_at_least(math.ceil(box[4 * d] / 0.1)) for d in range(3)]
    sim = GpuSimulation(system, {"alpha": ALPHA, "grid": grid, "pmeOrder": 4, "dispersionCorrection": False,
                                 "skin": 0.1, "waterSolver": 1})
    sim.setState(pos)
    sim.initialise()
    # a physical state: the seeded lattice minimised and run for 1,000 steps (on the raw
    # lattice the Coulomb terms cancel to a total ~600x smaller than themselves)
    sim.minimise(maxIterations=100, forceTolerance=1000.0)
    sim.run(1000, blockSize=100)
    held = sim.readState()["positions"].astype(np.float64)  # the f32 coordinates the device holds
    energy, forces = sim.debugEvaluate()
    expect, expect_forces = oracle.Oracle(system).potential(held, method="PME", alpha=ALPHA, grid=grid, order=4)
    terms = {
        "bonded": (energy["bonded"], expect["bonded"]),
        "lennardJones": (energy["lennard_jones"], expect["lennardJones"]),
        "coulombDirect": (energy["coulomb_direct"], expect["coulombDirect"]),
        "coulombReciprocal": (energy["coulomb_reciprocal"], expect["coulombReciprocal"]),
        "coulombSelf": (energy["coulomb_self"], expect["coulombSelf"] + expect["coulombNetCharge"]),
        "potential": (energy["potential"], expect["total"]),
    }
    errors = {k: abs(a - b) / max(abs(b), 1e-300) for k, (a, b) in terms.items()}
    print(f"absolute {n_atoms}: " + ", ".join(f"{k} {a:.6f} vs {b:.6f}" for k, (a, b) in terms.items()))
    diff = forces - expect_forces
    rms = math.sqrt(float(np.mean(expect_forces ** 2)))
    force_rms_error = math.sqrt(float(np.mean(diff ** 2))) / rms
    return errors, force_rms_error, float(np.max(np.abs(diff))) / rms


@pytest.mark.parametrize("n_atoms", [2854, 23558, 99999])
def test_every_energy_term_within_1e5_of_the_fp64_oracle(n_atoms):
    errors, force_rms_error, force_worst = precision_case(n_atoms)
    print(f"precision {n_atoms}: " + ", ".join(f"{k} {v:.2e}" for k, v in errors.items()) +
          f", force rms error {force_rms_error:.2e} of rms, worst {force_worst:.2e} of rms")
    for term, err in errors.items():
        assert err < 1e-5, (term, err)
    assert force_rms_error < 1e-5
    assert force_worst < 3e-3
