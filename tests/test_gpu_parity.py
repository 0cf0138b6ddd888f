"""Parity of the CUDA engine (through the C ABI) against the CPU oracle.

Bars follow the reference's own GPU differential checks (tools/gpu/check-*.mjs):
index structures bit-exact; energies per term relative to the FP64 oracle; forces as the
worst component error over the force rms; one integrator step with supplied noise.
"""
import math

import numpy as np
import pytest

import oracle
from goldens import system_for
from rainmd_b200 import synthetic
from rainmd_b200.simulation import BatchSimulation, GpuSimulation
from rainmd_b200.topology import build_system

pytestmark = pytest.mark.gpu

ALPHA = 2.6282608939112584


def relative(ours, theirs, floor=1.0):
    return abs(ours - theirs) / max(abs(theirs), floor)


def f32(positions):
    """The coordinates the device holds: forces are compared at the same inputs, so the
    f32 rounding of box-spanning coordinates (k*span*eps on a stiff bond) is not charged
    to the kernels (check-bonded.mjs:1-30)."""
    return np.asarray(positions, dtype=np.float32).astype(np.float64)


def oracle_terms(system, positions, alpha, grid, order):
    e, f = oracle.Oracle(system).potential(f32(positions), method="PME", alpha=alpha, grid=grid,
                                           order=order)
    return e, f


def engine_for(system, positions, **options):
    opts = {"alpha": ALPHA, "grid": [24, 24, 24], "skin": 0.1, "dispersionCorrection": False}
    opts.update(options)
    sim = GpuSimulation(system, opts)
    sim.setState(positions)
    sim.initialise()
    return sim


def symmetric_exclusions(system):
    n = system["topology"]["atomCount"]
    ex = system["exceptions"]
    a = np.concatenate([ex["atomA"], ex["atomB"]])
    b = np.concatenate([ex["atomB"], ex["atomA"]])
    order = np.lexsort((b, a))
    start = np.zeros(n + 1, np.int32)
    np.add.at(start, a + 1, 1)
    return np.cumsum(start).astype(np.int32), b[order].astype(np.int32)


@pytest.mark.parametrize("group", [4, 8, 16, 32])
@pytest.mark.parametrize("cutoff", [1.25, 1.0, 0.7, 0.5])
def test_cell_and_neighbour_lists_bit_exact(cutoff, group):
    """check-nonbonded.mjs:12-19, 240-262 at four cell geometries and every search-group
    size, compared bit for bit with the f32 restatement of the reference's assignment and
    search. This 1,190-atom box has few groups, so 4-atom groups take the split search (three
    warps a group, hits staged per x-slab); at 1.25 nm (2 x 2 x 1 cells) some atoms have more
    than 512 partners in one slab, which overflows the staging and takes its fallback."""
    s, pos, _ = system_for("ala-wat", cutoff=cutoff)
    sim = engine_for(s, pos, alpha=None, grid=None, neighbourGroupAtoms=group, pairList=1)
    counts, start, atoms = sim.debugCells()
    lc = np.float32(cutoff) + np.float32(0.1)
    P = oracle.pack_params(s["boxVectors"], cutoff, float(np.float32(cutoff + 0.1)), 1.0)
    coa, cs, ca = oracle.cell_list_f32(pos.astype(np.float32), P, counts)
    assert np.array_equal(start, cs)
    assert np.array_equal(atoms, ca)
    es, ep = symmetric_exclusions(s)
    cap, ncount, rows, required = sim.debugNeighbours()
    nb, nc, req = oracle.neighbour_list_f32(pos.astype(np.float32), P, counts, cs, ca, es, ep, cap)
    assert required == req
    assert np.array_equal(ncount, nc)
    for i in range(len(nc)):
        assert np.array_equal(rows[i, :nc[i]], nb[i, :nc[i]])
    del lc


def test_neighbour_overflow_grows_capacity():
    """check-capacity.mjs / check-nonbonded.mjs:54: a forced capacity of 64 is measured
    and grown, never silently truncated."""
    s, pos, _ = system_for("ala-wat")
    sim = engine_for(s, pos, maxNeighbours=64)
    d = sim.diagnostics()
    assert d["neighbour_growths"] >= 1
    assert d["neighbour_capacity"] >= d["neighbour_required"] > 64
    e = sim.energy()
    eo, _ = oracle_terms(s, pos, ALPHA, [24, 24, 24], 5)
    assert relative(e["lennardJones"], eo["lennardJones"]) < 1e-5


@pytest.mark.parametrize("constraints", ["HBonds", "none"])
def test_energies_and_forces_vs_oracle_order5(constraints):
    """check-forces.mjs:214-233 bars: bonded 1e-5, LJ 1e-5, Coulomb 2e-5, total 5e-5,
    forces 3e-3 of rms; here against the FP64 oracle at the OpenMM fixture's settings."""
    s, pos, raw = system_for("ala-wat", constraints=constraints, rigid_water=constraints != "none")
    sim = engine_for(s, pos)
    e, forces = sim.debugEvaluate()
    eo, fo = oracle_terms(s, pos, ALPHA, [24, 24, 24], 5)
    assert relative(e["bonded"], eo["bonded"]) < 1e-5
    assert relative(e["lennard_jones"], eo["lennardJones"]) < 1e-5
    assert relative(e["coulomb_direct"], eo["coulombDirect"]) < 2e-5
    assert relative(e["coulomb_reciprocal"], eo["coulombReciprocal"]) < 2e-5
    assert relative(e["coulomb_self"], eo["coulombSelf"] + eo["coulombNetCharge"]) < 1e-12
    assert relative(e["potential"], eo["total"]) < 5e-5
    rms = math.sqrt(np.mean(fo ** 2))
    assert np.max(np.abs(forces - fo)) / rms < 3e-3
    # and against OpenMM itself, through the oracle-pinned fixture
    ref = float(raw[f"{'ala-wat-pme' if constraints == 'HBonds' else 'ala-wat-pme-free'}:energy.total"])
    assert relative(e["potential"], ref) < 5e-5


@pytest.mark.parametrize("term", ["direct", "bonded", "reciprocal"])
@pytest.mark.parametrize("accumulation", [0, 1])
def test_force_terms_vs_oracle(term, accumulation):
    """Per-term forces. Direct space: 1e-4 of rms (check-nonbonded.mjs:283-298).
    Reciprocal: 3e-3 of rms (check-pme.mjs:173-178). Bonded: the f32 bound the reference
    derives for its bonded check (check-bonded.mjs:1-30), a few ulp of the bond length times
    the stiffest force constant."""
    s, pos, _ = system_for("ala-wat")
    sim = engine_for(s, pos, forceAccumulation=accumulation)
    got = sim.debugForceTerm(term)
    expect = oracle.Oracle(s).term_forces(f32(pos), term, alpha=ALPHA, grid=[24, 24, 24], order=5)
    assert np.all(np.isfinite(got))
    if term == "bonded":
        k_max = float(np.max(s["harmonicBonds"]["k"]))
        r_max = float(np.max(s["harmonicBonds"]["r0"]))
        assert np.max(np.abs(got - expect)) < k_max * r_max * 2.0 ** -22
    else:
        rms = math.sqrt(np.mean(expect ** 2))
        assert np.max(np.abs(got - expect)) / rms < (1e-4 if term == "direct" else 3e-3)


def test_energies_vs_oracle_order4_config0_shape():
    """The benchmark form: PME order 4, 24^3, cutoff 0.9 nm, on the 1190-atom synthetic box."""
    topo, pos = synthetic.config0(seed=1)
    s = build_system(topo, cutoff=0.9)
    alpha = oracle.alpha_from_tolerance(0.9, 5e-4)
    sim = GpuSimulation(s, {"pmeOrder": 4, "grid": [24, 24, 24], "skin": 0.1, "dispersionCorrection": False})
    sim.setState(pos)
    sim.initialise()
    e, forces = sim.debugEvaluate()
    eo, fo = oracle_terms(s, pos, alpha, [24, 24, 24], 4)
    assert relative(e["lennard_jones"], eo["lennardJones"]) < 1e-5
    assert relative(e["coulomb_direct"], eo["coulombDirect"]) < 2e-5
    assert relative(e["coulomb_reciprocal"], eo["coulombReciprocal"]) < 2e-5
    assert relative(e["bonded"], eo["bonded"]) < 1e-5
    rms = math.sqrt(np.mean(fo ** 2))
    assert np.max(np.abs(forces - fo)) / rms < 3e-3


def test_spread_grid_vs_oracle():
    """check-pme.mjs:173-178: the spread charge grid point by point, bar 1e-5."""
    s, pos, _ = system_for("ala-wat")
    sim = engine_for(s, pos)
    grid = sim.debugChargeGrid(points=24 ** 3)
    _, _, q = oracle.Oracle(s).reciprocal(pos, ALPHA, [24, 24, 24], 5, want_grid=True)
    assert np.max(np.abs(grid - q)) < 1e-5
    assert np.max(np.abs(grid)) < 128  # fixed-point headroom (pme.js:25-43)


@pytest.mark.parametrize("grid", [[24, 24, 24], [24, 32, 20], [27, 25, 16]])
def test_fft_round_trip_vs_dft(grid):
    """check-fft.mjs: the engine's R2C/C2R transform against a DFT on random data; bar
    20*sqrt(stages)*2^-24 relative to the spectrum scale."""
    s, pos, _ = system_for("ala-wat")
    sim = engine_for(s, pos, grid=grid)
    rng = np.random.default_rng(5)
    data = rng.normal(size=grid).reshape(-1)
    nx, ny, nz = grid
    half, back = sim.debugFft(data, nx * ny * (nz // 2 + 1))
    expect = np.fft.fftn(data.reshape(grid))[:, :, : nz // 2 + 1].reshape(-1)
    scale = np.max(np.abs(expect))
    stages = sum(math.ceil(math.log2(n)) for n in grid)
    assert np.max(np.abs(half - expect)) / scale < 20 * math.sqrt(stages) * 2 ** -24 * 8
    assert np.max(np.abs(back / (nx * ny * nz) - data)) < 1e-5


def test_one_integrator_step_with_supplied_noise():
    """check-integrator.mjs:68-127: one step with shared noise and shared forces; positions
    within 1e-5 nm and velocities within 1e-3 of their scale."""
    s, pos, _ = system_for("ala-wat")
    rng = np.random.default_rng(11)
    vel = rng.normal(scale=0.3, size=pos.size)
    o = oracle.Oracle(s)
    integ = o.integrator(timestep=0.002, temperature=300, friction=1.0, seed=3, tolerance=1e-5)
    # the device starts from f32 state; give the oracle the same rounded inputs
    pos32 = pos.astype(np.float32).astype(np.float64)
    sim = engine_for(s, pos32, temperature=300, friction=1.0, seed=3, tolerance=1e-5, timestep=0.002)
    noise = rng.normal(size=pos.size).astype(np.float32)
    sim.setState(pos32, vel.astype(np.float32).astype(np.float64), step=0, suppliedNoise=True)
    sim.setNoise(noise)
    sim.initialise()
    _, f_dev = sim.debugEvaluate()
    sim.run(1, blockSize=1)
    state = sim.readState()
    p1, v1, _ = o.langevin_step(pos32, vel.astype(np.float32).astype(np.float64), f_dev, integ, 0,
                                noise=noise.astype(np.float64))
    _, f1 = o.potential(p1, method="PME", alpha=ALPHA, grid=[24, 24, 24], order=5)
    v1 = o.finish_step(p1, v1, f1, integ)
    assert np.max(np.abs(state["positions"] - p1)) < 1e-5
    vscale = np.max(np.abs(v1))
    assert np.max(np.abs(state["velocities"] - v1)) < 1e-3 * vscale


def test_constraints_hold_and_temperature_is_sane():
    """check-integrator.mjs:137-252: constraint geometry after many steps < 2e-5 relative;
    the thermostat holds the temperature near its setpoint."""
    s, pos, _ = system_for("ala-wat")
    sim = engine_for(s, pos, temperature=300, seed=9, skin=0.15, rebuildInterval=10)
    sim.minimise(maxIterations=50)
    sim.run(400, blockSize=20)
    state = sim.readState()
    p = state["positions"].reshape(-1, 3).astype(np.float64)
    c = s["constraints"]
    lengths = np.linalg.norm(p[c["atomA"]] - p[c["atomB"]], axis=1)
    assert np.max(np.abs(lengths - c["distance"]) / c["distance"]) < 2e-5
    e = sim.energy()
    assert math.isfinite(e["potential"]) and math.isfinite(e["kinetic"])
    assert 200 < e["temperature"] < 400
    d = sim.diagnostics()
    # a violated skin is detected and answered by a shorter interval (simulation.js:544-623)
    assert d["skin_violations"] == 0 or d["rebuild_shrinks"] > 0
    assert not d["shake_hit_iteration_cap"]


def test_settle_keeps_rigid_water():
    """SETTLE (new work): the water triangle holds to 2e-5 while SHAKE handles the rest."""
    s, pos, _ = system_for("ala-wat")
    sim = engine_for(s, pos, waterSolver=1, temperature=300, seed=4, skin=0.15, rebuildInterval=10,
                     adaptiveRebuild=False)
    assert sim.diagnostics()["settle_count"] > 300
    sim.minimise(maxIterations=50)
    sim.run(300, blockSize=20)
    p = sim.readState()["positions"].reshape(-1, 3).astype(np.float64)
    c = s["constraints"]
    lengths = np.linalg.norm(p[c["atomA"]] - p[c["atomB"]], axis=1)
    assert np.max(np.abs(lengths - c["distance"]) / c["distance"]) < 2e-5
    assert 200 < sim.energy()["temperature"] < 400


def test_runs_are_bitwise_deterministic():
    """Fixed-point forces and the counter RNG: the same run twice gives the same bits."""
    s, pos, _ = system_for("ala-wat")
    out = []
    for _ in range(2):
        sim = engine_for(s, pos, seed=21, temperature=300, skin=0.15, rebuildInterval=5, adaptiveRebuild=False)
        sim.run(50, blockSize=10)
        out.append(sim.readState())
        sim.release()
    assert np.array_equal(out[0]["positions"], out[1]["positions"])
    assert np.array_equal(out[0]["velocities"], out[1]["velocities"])
    assert np.array_equal(out[0]["forces"], out[1]["forces"])


def test_resume_is_bitwise():
    """Checkpoint/resume: 40 steps equal 20 steps, read state, restore at step 20, 20 more.
    The restart rebuilds its list at a different step than the straight run did; per-pair
    fixed-point accumulation makes the forces independent of the neighbour-row order."""
    s, pos, _ = system_for("ala-wat")
    opts = dict(seed=5, temperature=300, skin=0.15, rebuildInterval=5, adaptiveRebuild=False)
    a = engine_for(s, pos, **opts)
    a.run(40, blockSize=10)
    full = a.readState()
    b = engine_for(s, pos, **opts)
    b.run(20, blockSize=10)
    mid = b.readState()
    c = engine_for(s, pos, **opts)
    c.setState(mid["positions"].astype(np.float64), mid["velocities"].astype(np.float64), step=20)
    c.initialise()
    c.run(20, blockSize=10)
    assert np.array_equal(c.readState()["positions"], full["positions"])


def test_batch_equals_separate_systems():
    """Batching changes nothing about a system's physics: energies match the solo run."""
    systems = synthetic.batch(3, low=1000, high=2500, seed=3)
    built = [build_system(t, cutoff=0.9) for t, _ in systems]
    opts = {"pmeOrder": 4, "skin": 0.1, "dispersionCorrection": True}
    batch = BatchSimulation(built, opts)
    for k, (_, pos) in enumerate(systems):
        batch.setState(k, pos)
    batch.initialise()
    for k, (t, pos) in enumerate(systems):
        solo = GpuSimulation(built[k], opts)
        solo.setState(pos)
        solo.initialise()
        eb, es = batch.energy(k), solo.energy()
        for key in ("lennardJones", "coulombDirect", "coulombReciprocal", "bonded", "potential"):
            assert eb[key] == es[key], key
        solo.release()


@pytest.mark.parametrize("scale", ["0.97", "1.00", "1.02"])
def test_scale_volume_vs_openmm(scale):
    """check-barostat.mjs:41-69: the energy at a forced scale vs OpenMM, bar 5e-5."""
    s, pos, raw = system_for("ala-wat")
    sim = engine_for(s, pos, dispersionCorrection=True)
    energy = sim.scaleVolume(float(scale))
    ref = float(raw[f"ala-wat-scale-{scale}:energy.total"])
    assert relative(energy, ref) < 5e-5


def test_barostat_moves_and_accepts():
    """check-barostat.mjs:97-105: moves are attempted on the device, some accepted, the
    volume changes and the acceptance stays in (0.05, 0.95)."""
    s, pos, _ = system_for("ala-wat")
    sim = engine_for(s, pos, pressure=1.0, barostatInterval=10, temperature=300, seed=2, skin=0.15,
                     rebuildInterval=10, adaptiveRebuild=False, dispersionCorrection=True)
    sim.minimise(maxIterations=30)
    v0 = sim.energy()["volume"]
    sim.run(600, blockSize=10)
    d = sim.diagnostics()
    assert d["barostat_attempts"] >= 50
    assert 0.05 < d["barostat_accepted"] / d["barostat_attempts"] < 0.95
    assert sim.energy()["volume"] != v0


def test_restraint_vs_openmm():
    s, _, raw = system_for("ala-wat")
    pos = raw["ala-wat-restraint-500:positions"].reshape(-1)
    atoms = raw["ala-wat-restraint-500:restraint.atoms"]
    reference = system_for("ala-wat")[1]
    sim = engine_for(s, pos, restraintForce=float(raw["ala-wat-restraint-500:restraint.force"]),
                     restraintAtoms=atoms, restraintReference=reference)
    e, _ = sim.debugEvaluate()
    assert relative(e["position_restraint"], float(raw["ala-wat-restraint-500:group.CustomExternalForce"])) < 1e-5
    assert relative(e["potential"], float(raw["ala-wat-restraint-500:energy.total"])) < 5e-5


def test_fused_and_separate_reciprocal_passes_agree():
    """A system with a small kz plane (up to 52 x 52 points) takes the fused y-x-convolve-x-y
    pass one block a plane; larger planes up to 128 x 128 take it one thread-block cluster a
    plane, rows and columns split four ways (evenly, or raggedly as 54 = 14 + 14 + 14 + 12);
    a 160 x 160 plane takes the separate passes. In one batch each gives its solo energies bit
    for bit, and all match the FP64 oracle's reciprocal energy and forces."""
    s, pos, _ = system_for("ala-wat")
    grids = ([24, 24, 24], [54, 60, 20], [72, 54, 20], [120, 120, 24], [160, 160, 16])
    solo = []
    for grid in grids:
        sim = engine_for(s, pos, grid=grid)
        e, forces = sim.debugEvaluate()
        eo, fo = oracle_terms(s, pos, ALPHA, grid, 5)
        assert relative(e["coulomb_reciprocal"], eo["coulombReciprocal"]) < 2e-5, grid
        rms = math.sqrt(np.mean(fo ** 2))
        assert np.max(np.abs(forces - fo)) / rms < 3e-3, grid
        solo.append(e)
        sim.release()
    batch = BatchSimulation([s] * len(grids), [{"alpha": ALPHA, "grid": g, "skin": 0.1,
                                                 "dispersionCorrection": False} for g in grids])
    for k in range(len(grids)):
        batch.setState(k, pos)
    batch.initialise()
    for k in range(len(grids)):
        e, _ = batch.debugEvaluate(k)
        for key in ("coulomb_reciprocal", "potential"):
            assert e[key] == solo[k][key], (k, key)
