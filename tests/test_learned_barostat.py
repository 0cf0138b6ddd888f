"""The learned barostat: the device network against the CPU oracle (forward pass and
gradients), and the two-stage delayed-acceptance barostat against the plain exact one
(what the trained network saves, and that the density it samples is the same)."""
import math

import numpy as np
import pytest

from oracle import surrogate as sg
from rainmd_b200 import synthetic
from rainmd_b200.simulation import GpuSimulation, surrogate_evaluate
from rainmd_b200.topology import build_system

pytestmark = pytest.mark.gpu


def test_device_forward_matches_oracle():
    rng = np.random.default_rng(2)
    params = sg.random_parameters(seed=2)
    x = rng.normal(size=(64, 8)).astype(np.float32)
    out, _, _ = surrogate_evaluate(params, x)
    ref = sg.forward(params, x)[0]
    assert np.max(np.abs(out - ref)) < 1e-5 * max(1.0, np.max(np.abs(ref)))


@pytest.mark.parametrize("count", [64, 17, 1])
def test_device_gradients_match_oracle(count):
    rng = np.random.default_rng(count)
    params = sg.random_parameters(seed=count)
    x = rng.normal(size=(count, 8)).astype(np.float32)
    t = (rng.normal(size=count) * 0.5).astype(np.float32)
    _, grads, loss = surrogate_evaluate(params, x, t, gradients=True)
    ref_loss, ref = sg.loss_and_gradients(params, x, t)
    assert abs(loss - ref_loss) <= 1e-5 * max(1.0, ref_loss)
    for lo, hi in ((sg.W1, sg.B1), (sg.B1, sg.W2), (sg.W2, sg.B2), (sg.B2, sg.W3), (sg.W3, sg.B3), (sg.B3, sg.PARAMS)):
        err = np.linalg.norm(grads[lo:hi] - ref[lo:hi])
        assert err <= 1e-4 * np.linalg.norm(ref[lo:hi]) + 1e-7, (lo, err)


def _without_lj(system):
    """Coulomb and bonded terms only: no energy jump where pairs cross a truncated LJ
    cutoff, so the finite difference measures the virial alone."""
    s = dict(system)
    s["topology"] = dict(system["topology"])
    s["topology"]["ljA"] = np.zeros_like(np.asarray(system["topology"]["ljA"], dtype=float))
    s["topology"]["ljB"] = np.zeros_like(np.asarray(system["topology"]["ljB"], dtype=float))
    s["exceptions"] = dict(system["exceptions"])
    s["exceptions"]["ljA"] = np.zeros_like(np.asarray(system["exceptions"]["ljA"], dtype=float))
    s["exceptions"]["ljB"] = np.zeros_like(np.asarray(system["exceptions"]["ljB"], dtype=float))
    return s


@pytest.mark.parametrize("kind", ["water", "chain"])
def test_volume_derivative_matches_finite_difference(kind):
    """dU/dlnV for rigid molecular scaling (atomic virial of every term, the reciprocal-space
    sum and the molecular correction) against a central difference of scaleVolume."""
    if kind == "water":
        topo, pos = synthetic.water_box(2854, seed=5)
        grid = [32, 32, 32]
    else:
        topo, pos = synthetic.config0(seed=5)
        grid = [24, 24, 24]
    system = _without_lj(build_system(topo, cutoff=0.9))
    sim = GpuSimulation(system, {"alpha": 3.85, "grid": grid, "pmeOrder": 4, "dispersionCorrection": False,
                                 "skin": 0.1, "temperature": 300.0})
    sim.setState(pos)
    sim.initialise()
    derivative = sim.energy()["volumeDerivative"]
    eps = 1e-3
    up = sim.scaleVolume((1 + eps) ** (1 / 3))
    down = sim.scaleVolume(((1 - eps) / (1 + eps)) ** (1 / 3))
    fd = (up - down) / math.log((1 + eps) / (1 - eps))
    assert abs(fd - derivative) <= 0.02 * abs(fd) + 1.0, (fd, derivative)


def _npt_density(learned, moves, seed, warmup=100):
    topo, pos = synthetic.water_box(2854, seed=11)
    system = build_system(topo, cutoff=0.9)
    sim = GpuSimulation(system, {"pmeOrder": 4, "grid": [32, 32, 32], "temperature": 300.0, "pressure": 1.0,
                                 "barostatInterval": 25, "seed": seed, "waterSolver": 1,
                                 "learnedBarostat": 1 if learned else 0, "learnedWarmupMoves": warmup})
    sim.setState(pos)
    sim.initialise()
    sim.minimise(maxIterations=200)
    sim.run(2500)
    mass = float(np.sum(system["topology"]["masses"]))
    volumes = []
    for _ in range(moves):
        sim.run(25)
        volumes.append(sim.diagnostics()["volume"])
    density = mass / np.array(volumes) * 1.66053906660  # amu/nm^3 -> kg/m^3
    kept = density[moves // 5:]
    blocks = np.array([b.mean() for b in np.array_split(kept, 20)])
    return kept.mean(), blocks.std(ddof=1) / math.sqrt(len(blocks)), sim


def test_learned_barostat_saves_exact_evaluations_and_keeps_the_density():
    """What the trained network gains: after its warm-up, stage 1 rejects most moves without an
    exact trial evaluation, while delayed acceptance keeps the NPT density of the plain exact
    barostat (same system, seed and length; block-averaged standard errors)."""
    moves, warmup = 2000, 100
    plain, plain_se, plain_sim = _npt_density(False, moves, seed=7, warmup=warmup)
    learned, learned_se, sim = _npt_density(True, moves, seed=7, warmup=warmup)
    report = sim.surrogateReport()
    assert report["screening"] == 1
    assert report["prediction_error_kT"] < 1.0
    after = report["attempts"] - warmup
    exact_after = report["exact_evaluations"] - warmup
    saved = 1.0 - exact_after / after
    assert saved >= 0.5, saved
    assert plain_sim.diagnostics()["barostat_exact_evaluations"] == plain_sim.diagnostics()["barostat_attempts"]
    sigma = math.hypot(plain_se, learned_se)
    assert abs(learned - plain) < 3.0 * sigma, (plain, plain_se, learned, learned_se)
