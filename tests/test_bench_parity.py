"""Parity on the benchmark's own configuration, through the C ABI.

The benchmark runs the 23,558-atom TIP3P box (rc 0.9 nm, skin 0.25 nm, PME order 4 on 64^3)
with autotuned launch shapes and lists rebuilt on demand inside the step graph. Here:
  - the cell and neighbour lists the device holds after on-demand rebuilds mid-run equal, bit
    for bit, the f32 restatement of the reference's cell assignment and search
    (cell-list.js:43-176, neighbours.js:46-151) run on the positions the lists were built from,
    with the cell counts from the oracle's planCellList (cells.js:101-171), not from the device;
    for the autotuned search shape and for the one-warp 4- and 16-atom searches, and for every
    system of a batch;
  - the thermostat's draws on the device equal uniformAt (shared/random.js:59) bit for bit, and
    its normals gaussianTriple (random.js:66-87) to f32 rounding; one integrator step with the
    device's own noise matches the oracle's step with the oracle's own draws;
  - every volume move's proposal, Metropolis weight and decision equal the FP64 restatement of
    attemptVolumeChange (webgpu/simulation.js:995-1070; metropolisWeight, barostat.js:158-162),
    an accepted move keeps the scaled state and a rejected move restores the old one bitwise;
  - a non-finite state ends a run with NonFiniteStateError (shared/finite.js:63-95).
"""
import math

import numpy as np
import pytest

import oracle
from goldens import system_for
from rainmd_b200 import synthetic
from rainmd_b200.simulation import BatchSimulation, GpuSimulation, NonFiniteStateError, planSystem
from rainmd_b200.topology import build_system

pytestmark = pytest.mark.gpu

BOLTZMANN = 0.008314462618      # shared/units.js:50
BAR = 0.06022140857             # kJ/mol/nm^3 per bar, shared/units.js:53


BENCH_SKIN = 0.25      # bench.py LIST_SKIN: the water boxes
SMALL_BOX_SKIN = 0.15  # bench.py SMALL_BOX_SKIN: the 1,190-atom system and the batch


def bench_options(grid, seed=7, skin=BENCH_SKIN, **extra):
    """The benchmark's options (bench.py options_for)."""
    o = {"timestep": 0.002, "temperature": 300.0, "friction": 1.0, "seed": seed, "pmeOrder": 4,
         "grid": grid, "ewaldTolerance": 5e-4, "waterSolver": 1, "skin": skin, "rebuildInterval": 10,
         "adaptiveRebuild": True, "dispersionCorrection": True}
    o.update(extra)
    return o


def water(n, seed=1):
    topo, pos = synthetic.water_box(n, seed=seed)
    system = build_system(topo, cutoff=0.9)
    box = system["boxVectors"]
    grid = [smooth(math.ceil(box[4 * d] / 0.1)) for d in range(3)]
    return system, pos, grid


def chain1190(seed=1):
    topo, pos = synthetic.config0(seed=seed)
    return build_system(topo, cutoff=0.9), pos, [24, 24, 24]


def smooth(n):
    while True:
        r = n
        for p in (2, 3, 5):
            while r % p == 0:
                r //= p
        if r == 1:
            return n
        n += 1


def exclusion_gather(system):
    """buildExclusionGather (cells.js:191-227): every excluded pair in both directions, each
    atom's partners sorted."""
    t = system["topology"]
    n = t["atomCount"]
    start, partners = np.asarray(t["exclusions"]["start"]), np.asarray(t["exclusions"]["partners"])
    a = np.repeat(np.arange(n), np.diff(start[: n + 1]))
    b = partners[: len(a)]
    left, right = np.concatenate([a, b]), np.concatenate([b, a])
    order = np.lexsort((right, left))
    counts = np.bincount(left, minlength=n)
    out_start = np.zeros(n + 1, np.int32)
    out_start[1:] = np.cumsum(counts)
    return out_start, right[order].astype(np.int32)


def assert_lists_match_oracle(sim, system, index=0, skin=0.15):
    """The device's cell and neighbour lists against the oracle's, from the positions the
    device built them from and the cell counts planCellList gives."""
    n = system["topology"]["atomCount"]
    box = system["boxVectors"]
    cutoff = system["options"]["cutoff"]
    plan = oracle.plan_cell_list(n, box, cutoff, skin=skin)
    origin = sim.debugRead("list_origin", 3 * n, index).astype(np.float32)
    counts, start, atoms = sim.debugCells(index)
    assert counts == plan["counts"]
    P = oracle.pack_params(box, cutoff, float(np.float32(cutoff + skin)), 1.0)
    _, cs, ca = oracle.cell_list_f32(origin, P, plan["counts"])
    assert np.array_equal(start, cs)
    assert np.array_equal(atoms, ca)
    es, ep = exclusion_gather(system)
    cap, ncount, rows, required = sim.debugNeighbours(index)
    nb, nc, req = oracle.neighbour_list_f32(origin, P, plan["counts"], cs, ca, es, ep, cap)
    assert required == req
    assert np.array_equal(ncount, nc)
    used = np.arange(cap)[None, :] < nc[:, None]
    assert np.array_equal(np.where(used, rows, 0), np.where(used, nb, 0))
    return int(nc.sum())


def assert_group_rows_cover(sim, system, index=0, skin=0.15):
    """The group-pair rows the device holds, expanded to atom pairs, against the oracle's rows
    from the positions they were built from: every non-excluded pair within the list cutoff is
    listed, through an image within the list cutoff, exactly once unless the box has fewer than
    three cells on an axis (then once per image within the list cutoff of the group); no
    excluded pair and no atom with itself is listed. Returns the number of listed pairs."""
    n = system["topology"]["atomCount"]
    box = np.asarray(system["boxVectors"], dtype=np.float64)
    cutoff = system["options"]["cutoff"]
    plan = oracle.plan_cell_list(n, box, cutoff, skin=skin)
    origin = sim.debugRead("list_origin", 3 * n, index).astype(np.float32)
    P = oracle.pack_params(box, cutoff, float(np.float32(cutoff + skin)), 1.0)
    _, cs, ca = oracle.cell_list_f32(origin, P, plan["counts"])
    es, ep = exclusion_gather(system)
    nb, nc, _ = oracle.neighbour_list_f32(origin, P, plan["counts"], cs, ca, es, ep, 4096)
    rows = np.repeat(np.arange(n), nc)
    cols = nb[np.arange(4096)[None, :] < nc[:, None]]
    expect = np.unique(np.minimum(rows, cols).astype(np.int64) * n + np.maximum(rows, cols))
    g = sim.debugGroupRows(index)
    cap = g["capacity"]
    used = np.arange(cap)[None, :] < g["counts"][:, None]
    q_idx, k_idx = np.nonzero(used)
    partner, code, mask = g["partners"][q_idx, k_idx], g["codes"][q_idx, k_idx], g["masks"][q_idx, k_idx]
    pairs_i, pairs_j, pairs_code = [], [], []
    for a in range(4):
        atom = g["atoms"][q_idx, a]
        keep = (atom >= 0) & (((mask >> a) & 1) == 0)
        pairs_i.append(atom[keep])
        pairs_j.append(partner[keep])
        pairs_code.append(code[keep])
    pi, pj, pc = np.concatenate(pairs_i), np.concatenate(pairs_j), np.concatenate(pairs_code)
    assert not np.any(pi == pj)
    key = np.minimum(pi, pj).astype(np.int64) * n + np.maximum(pi, pj)
    excluded = np.unique(np.minimum(np.repeat(np.arange(n), np.diff(es)), ep).astype(np.int64) * n +
                         np.maximum(np.repeat(np.arange(n), np.diff(es)), ep))
    assert not np.any(np.isin(key, excluded))
    listed = np.unique(key)
    assert np.all(np.isin(expect, listed))
    stencil = all(c >= 3 for c in plan["counts"])
    if stencil:
        assert len(listed) == len(key)  # each pair once
    # the listed image of every pair within the list cutoff is one within it; image codes refer
    # to the positions wrapped into the box at the build (whole box vectors subtracted)
    ka, kb, kc = pc // 9 - 1, (pc // 3) % 3 - 1, pc % 3 - 1
    shift = (ka[:, None] * box[0:3] + kb[:, None] * box[3:6] + kc[:, None] * box[6:9])
    rows3 = box.reshape(3, 3)
    x = origin.astype(np.float64).reshape(-1, 3)
    x = x - np.floor(x @ np.linalg.inv(rows3)) @ rows3
    d2 = np.sum((x[pi] - x[pj] - shift) ** 2, axis=1)
    within = np.isin(key, expect)
    lc = cutoff + skin
    best = np.full(len(listed), np.inf)
    np.minimum.at(best, np.searchsorted(listed, key[within]), d2[within])
    assert np.all(best[np.isin(listed, expect)] <= lc * lc * 1.0002)
    return int(len(key))


@pytest.fixture(scope="module")
def bench_box():
    system, pos, grid = water(23558)
    probe = GpuSimulation(system, bench_options(grid))
    probe.setState(pos)
    probe.initialise()
    probe.minimise(maxIterations=50, forceTolerance=1000.0)
    relaxed = probe.readState()["positions"].astype(np.float64)
    probe.release()
    return system, relaxed, grid


@pytest.mark.parametrize("form,group", [(2, None), (1, None), (1, 4), (1, 16)])
def test_benchmark_lists_bit_exact_after_on_demand_rebuilds(bench_box, form, group):
    """23,558 atoms, 5^3 cells (the shifted stencil and bounding-box culls), ~6,000 4-atom groups
    (the one-warp search, not the split one) or the autotuned shape; the lists compared are the
    ones the IF node of the step graph last rebuilt, mid-run. With pair_list 2 the same builds
    wrote the group-pair rows the pair kernel walks: they cover every pair of the per-atom
    rows once."""
    system, pos, grid = bench_box
    options = bench_options(grid, pairList=form)
    if group is not None:
        options["neighbourGroupAtoms"] = group
    sim = GpuSimulation(system, options)
    sim.setState(pos)
    sim.initialise()
    builds0 = sim.diagnostics()["list_builds"]
    sim.run(150, blockSize=50)
    d = sim.diagnostics()
    assert d["rebuild_on_demand"] == 1
    assert d["list_builds"] - builds0 >= 3  # rebuilt on demand inside the graphs
    if group is not None:
        assert sim.kernelShapes()["neighbourGroupAtoms"] == group
    pairs = assert_lists_match_oracle(sim, system, skin=BENCH_SKIN)
    assert pairs > 23558 * 400
    if form == 2:
        assert assert_group_rows_cover(sim, system, skin=BENCH_SKIN) >= pairs // 2
    sim.release()


@pytest.mark.parametrize("cutoff", [1.25, 1.0, 0.7, 0.5])
def test_group_rows_cover_every_pair(cutoff):
    """The 1,190-atom fixture at four cutoffs: 2 x 2 x 1 cells (every image of a partner searched)
    to 5^3 (the stencil), the chain's exclusions masked."""
    s, pos, _ = system_for("ala-wat", cutoff=cutoff)
    sim = GpuSimulation(s, {"skin": 0.1, "dispersionCorrection": False, "pairList": 0})
    sim.setState(pos)
    sim.initialise()
    assert assert_group_rows_cover(sim, s, skin=0.1) > 0
    sim.release()


def test_batch_lists_bit_exact_per_system(bench_box):
    """One batch of three uneven systems (a 1,190-atom chain system and a 2,854-atom box with 2^3
    cells, the 23,558-atom box with 5^3): each system's lists after on-demand, per-system
    rebuilds equal the oracle's for that system alone."""
    items = [chain1190(), water(2854), bench_box]
    systems = [s for s, _, _ in items]
    batch = BatchSimulation(systems, [bench_options(g, seed=5 + k, skin=SMALL_BOX_SKIN, pairList=2)
                                      for k, (_, _, g) in enumerate(items)])
    for k, (_, p, _) in enumerate(items):
        batch.setState(k, p)
    batch.initialise()
    batch.minimise(maxIterations=30, forceTolerance=1000.0)
    batch.run(120, blockSize=40)
    for k, system in enumerate(systems):
        assert_lists_match_oracle(batch, system, index=k)
        assert_group_rows_cover(batch, system, index=k)
    batch.release()


def test_cell_plan_is_the_engines(bench_box):
    """The engine plans with the host code rmd_plan_system exposes: skin, cell counts, capacity,
    alpha and grid agree with the plan and with planCellList (per-atom rows, whose longest row
    planCellList's capacity covers; a group-pair row may be longer and grow it by grownPlan)."""
    system, pos, grid = bench_box
    options = bench_options(grid, pairList=1)
    sim = GpuSimulation(system, options)
    sim.setState(pos)
    sim.initialise()
    d = sim.diagnostics()
    plan = planSystem(system, options)
    expect = oracle.plan_cell_list(23558, system["boxVectors"], 0.9, skin=BENCH_SKIN)
    assert d["skin"] == plan["skin"] == BENCH_SKIN
    assert list(d["cell_counts"]) == plan["counts"] == expect["counts"]
    assert d["neighbour_capacity"] == plan["capacity"] == (expect["maxNeighbours"] + 3) // 4 * 4
    assert d["pme_alpha"] == plan["alpha"] and list(d["pme_grid"]) == plan["grid"] == grid
    sim.release()


@pytest.mark.parametrize("form", [1, 0])
def test_capacity_grows_by_grown_plan(form):
    """A forced capacity of 64 on the 1,190-atom fixture overflows at the first build; the engine
    grows it once by grownPlan (cells.js:282-288) from the measured requirement: the longest
    per-atom row (the oracle's), or with group-pair rows the longest group row."""
    s, pos, _ = system_for("ala-wat")
    sim = GpuSimulation(s, {"alpha": 2.6282608939112584, "grid": [24, 24, 24], "skin": 0.1,
                            "dispersionCorrection": False, "maxNeighbours": 64, "pairList": form})
    sim.setState(pos)
    sim.initialise()
    d = sim.diagnostics()
    assert d["neighbour_growths"] == 1
    if form == 1:
        P = oracle.pack_params(s["boxVectors"], 1.0, float(np.float32(1.1)), 1.0)
        plan = oracle.plan_cell_list(s["topology"]["atomCount"], s["boxVectors"], 1.0, skin=0.1)
        _, cs, ca = oracle.cell_list_f32(pos.astype(np.float32), P, plan["counts"])
        es, ep = exclusion_gather(s)
        _, _, req = oracle.neighbour_list_f32(pos.astype(np.float32), P, plan["counts"], cs, ca, es, ep, 2048)
    else:
        req = int(sim.debugGroupRows()["counts"].max())
        assert d["neighbour_required"] == req
    assert d["neighbour_capacity"] == (oracle.grown_plan(64, req) + 3) // 4 * 4
    sim.release()


@pytest.mark.parametrize("seed", [0, 3, 0x5a17, 0xdeadbeef])
@pytest.mark.parametrize("step", [0, 1, 4097, 2 ** 31 + 7])
def test_device_draws_match_uniform_at(seed, step):
    """uniformAt keeps the top 23 bits of the hash, so (s >> 9) + 0.5 scaled by 2^-23 is exact in
    f32: the device's uniforms equal the FP64 oracle's bit for bit. The normals are the f32
    Box-Muller triple; f32 log, sqrt and sincospi against their f64 counterparts stay within
    2e-5 absolute for |g| up to ~6."""
    from rainmd_b200.simulation import deviceDraws

    atom0, count = 1000, 3000
    u, g = deviceDraws(seed, atom0, count, step)
    expect_u = np.array([[oracle.uniform_at(seed, atom0 + k, step, c) for c in range(4)] for k in range(count)])
    assert np.array_equal(u.astype(np.float64), expect_u)
    expect_g = np.array([oracle.gaussian_triple(seed, atom0 + k, step) for k in range(count)])
    assert np.max(np.abs(g - expect_g)) < 2e-5


def test_one_integrator_step_with_device_noise():
    """check-integrator.mjs:68-127 with the thermostat's own draws on both sides: the device
    step (noise from (seed, atom, step)) against the oracle's langevinStep drawing
    gaussianTriple(seed, atom, step); positions within 1e-5 nm, velocities within 1e-3 of their
    scale."""
    s, pos, _ = system_for("ala-wat")
    rng = np.random.default_rng(12)
    vel = rng.normal(scale=0.3, size=pos.size)
    o = oracle.Oracle(s)
    integ = o.integrator(timestep=0.002, temperature=300, friction=1.0, seed=5, tolerance=1e-5)
    pos32 = pos.astype(np.float32).astype(np.float64)
    vel32 = vel.astype(np.float32).astype(np.float64)
    sim = GpuSimulation(s, {"alpha": 2.6282608939112584, "grid": [24, 24, 24], "skin": 0.1,
                            "dispersionCorrection": False, "temperature": 300, "friction": 1.0, "seed": 5,
                            "tolerance": 1e-5, "timestep": 0.002})
    sim.setState(pos32, vel32, step=17)
    sim.initialise()
    _, f_dev = sim.debugEvaluate()
    sim.run(1, blockSize=1)
    state = sim.readState()
    p1, v1, _ = o.langevin_step(pos32, vel32, f_dev, integ, 17, noise=None)
    _, f1 = o.potential(p1, method="PME", alpha=2.6282608939112584, grid=[24, 24, 24], order=5)
    v1 = o.finish_step(p1, v1, f1, integ)
    assert np.max(np.abs(state["positions"] - p1)) < 1e-5
    assert np.max(np.abs(state["velocities"] - v1)) < 1e-3 * np.max(np.abs(v1))
    sim.release()


def test_barostat_decisions_match_attempt_volume_change():
    """Twelve volume moves on the 1,190-atom fixture at 1 bar: the proposal is
    volumeScale * 2 * (uniformAt(seed ^ 0x5a17, attempt, 0, 0) - 0.5), the length scale its
    cube root, the weight metropolisWeight(dE, dV, V'/V) with N_mol kT ln(V'/V), and the move is
    accepted iff weight <= 0 or uniformAt(seed ^ 0x5a17, attempt, 1, 0) < exp(-weight / kT). An
    accepted move leaves the molecule-scaled positions and the scaled box; a rejected one leaves
    the old positions and box bit for bit."""
    s, pos, _ = system_for("ala-wat")
    seed, temperature, pressure = 21, 300.0, 1.0
    sim = GpuSimulation(s, {"alpha": 2.6282608939112584, "grid": [24, 24, 24], "skin": 0.15,
                            "dispersionCorrection": True, "temperature": temperature, "seed": seed,
                            "pressure": pressure, "barostatInterval": 25})
    sim.setState(pos)
    sim.initialise()
    sim.minimise(maxIterations=30)
    sim.run(50, blockSize=25)
    kT = BOLTZMANN * temperature
    molecules = s["molecules"]["count"]
    o = oracle.Oracle(s)
    outcomes = []
    for _ in range(12):
        sim.run(10, blockSize=10)
        before = sim.readState()
        d0 = sim.diagnostics()
        attempt = d0["barostat_attempts"] + 1
        scale = d0["volume_scale"] if d0["volume_scale"] > 0 else 0.01 * before["volume"]
        e0 = sim.energy()["potential"]
        move = sim.attemptVolumeChange()
        after = sim.readState()
        u0 = oracle.uniform_at(seed ^ 0x5a17, attempt, 0, 0)
        dv = scale * 2.0 * (u0 - 0.5)
        assert move["delta_volume"] == pytest.approx(dv, rel=1e-14, abs=1e-18)
        v0 = before["volume"]
        assert move["length_scale"] == pytest.approx(np.cbrt((v0 + dv) / v0), rel=1e-14)
        assert move["old_potential"] == pytest.approx(e0, rel=1e-12)
        w = oracle.metropolis_weight(move["new_potential"] - move["old_potential"], dv, (v0 + dv) / v0,
                                     pressure * BAR, kT, molecules)
        assert move["weight"] == pytest.approx(w, rel=1e-9, abs=1e-9)
        u1 = oracle.uniform_at(seed ^ 0x5a17, attempt, 1, 0)
        accept = w <= 0 or u1 < math.exp(-w / kT)
        assert bool(move["accepted"]) == accept
        ls = move["length_scale"]
        if accept:
            assert np.allclose(after["boxVectors"], before["boxVectors"] * ls, rtol=1e-15, atol=0)
            expect = o.scale_molecules(before["positions"].astype(np.float64), ls)
            assert np.max(np.abs(after["positions"] - expect)) < 2e-6
            # the trial energy is the potential of the scaled state (the PME grid stays fixed)
            scaled_system = dict(s)
            scaled_system["boxVectors"] = np.array(after["boxVectors"], dtype=np.float64)
            o2 = oracle.Oracle(scaled_system)
            scaled, _ = o2.potential(after["positions"].astype(np.float64), method="PME",
                                     alpha=2.6282608939112584, grid=[24, 24, 24], order=5)
            assert move["new_potential"] == pytest.approx(
                scaled["total"] + o2.dispersion(after["volume"], 1.0), rel=5e-5)
        else:
            assert np.array_equal(after["positions"], before["positions"])
            assert np.array_equal(after["boxVectors"], before["boxVectors"])
        outcomes.append(accept)
    assert any(outcomes) and not all(outcomes)
    sim.release()


def test_non_finite_state_raises():
    """A coordinate that is not a number makes the run stop with NonFiniteStateError at the
    end of the block (shared/finite.js:63-95; simulation.js:562-580). Every index the kernels
    derive from a coordinate is clamped (cell coordinates) or wrapped (PME grid points), so the
    non-finite value only travels through arithmetic."""
    s, pos, _ = system_for("ala-wat")
    sim = GpuSimulation(s, {"alpha": 2.6282608939112584, "grid": [24, 24, 24], "skin": 0.1,
                            "dispersionCorrection": False, "temperature": 300.0, "seed": 1})
    bad = np.array(pos, dtype=np.float64)
    bad[3 * 500 + 1] = np.nan
    sim.setState(bad)
    sim.initialise()
    with pytest.raises(NonFiniteStateError):
        sim.run(20, blockSize=10)
    sim.release()


@pytest.mark.parametrize("which", ["chain-1190", "water-23558"])
def test_moves_inside_step_graphs_evaluate_the_trial_state(which, bench_box):
    """Volume moves inside the step graphs are evaluated on the current lists when the
    displacement check, with the move's allowance, still trusts them (the atoms' wraps and
    origins scaled with them): each move's trial energy must be the oracle's potential of the
    molecule-scaled state in the scaled box (5e-5), in a 2 x 2 x 2-cell box (every image searched)
    and a 5^3 stencil box; an accepted move leaves the scaled box, a rejected one the old."""
    if which == "chain-1190":
        system, pos, grid = chain1190()
    else:
        system, pos, grid = bench_box
    skin = SMALL_BOX_SKIN if which == "chain-1190" else BENCH_SKIN
    sim = GpuSimulation(system, bench_options(grid, seed=13, skin=skin, pressure=1.0, barostatInterval=25))
    sim.setState(pos)
    sim.initialise()
    sim.minimise(maxIterations=30, forceTolerance=1000.0)
    sim.run(100, blockSize=25)
    alpha = oracle.alpha_from_tolerance(0.9, 5e-4)
    outcomes = []
    for _ in range(6):
        before = sim.readState()
        attempts = sim.diagnostics()["barostat_attempts"]
        sim.run(25, blockSize=25)
        assert sim.diagnostics()["barostat_attempts"] == attempts + 1
        move = sim.lastVolumeMove()
        after_box = np.asarray(sim.readState()["boxVectors"])
        ls = move["length_scale"]
        scaled_system = dict(system)
        scaled_system["boxVectors"] = np.asarray(before["boxVectors"], dtype=np.float64) * ls
        o = oracle.Oracle(scaled_system)
        scaled = oracle.Oracle(system).scale_molecules(before["positions"].astype(np.float64), ls)
        e, _ = o.potential(scaled.astype(np.float32).astype(np.float64), method="PME", alpha=alpha, grid=grid,
                           order=4)
        volume = float(np.prod(np.diag(np.asarray(scaled_system["boxVectors"]).reshape(3, 3))))
        expect = e["total"] + o.dispersion(volume, 0.9)
        assert move["new_potential"] == pytest.approx(expect, rel=5e-5), (which, move)
        if move["accepted"]:
            assert np.allclose(after_box, np.asarray(before["boxVectors"]) * ls, rtol=1e-15, atol=0)
        else:
            assert np.array_equal(after_box, np.asarray(before["boxVectors"]))
        outcomes.append(bool(move["accepted"]))
    sim.release()
