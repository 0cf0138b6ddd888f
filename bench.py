"""Benchmark: ns/day of the MD step on B200, and the reference CPU path beside it.

Workload (default): a 23,558-atom TIP3P water box at 0.997 g/cm^3 (7852 rigid waters plus
Na+ and Cl-), NVT at 300 K with 1/ps friction, 2 fs, 0.9 nm cutoff, PME order 4 on a 64^3
grid (<= 1 Å spacing), Ewald tolerance 5e-4, FP32 arithmetic with 64-bit fixed-point force
accumulation. Seeded synthetic coordinates stand in for the benchmark's structure files.

One bench "step" is one MD time step. The timed region is K steps run as CUDA-graph blocks
through the engine's public run path; each block is bracketed by CUDA events on the engine's
own stream and L2 is flushed (256 MB written) before every block, outside the events.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload ...]

Under torchrun each rank advances its own independent replica (the single-system path does
not shard); `value` is the aggregate over ranks, timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

TIMESTEP_PS = 0.002
METRIC = "ns/day (single system and batched aggregate) vs plain path at fixed energy error"


def ns_per_day(seconds_per_step: float, timestep_ps: float = TIMESTEP_PS) -> float:
    return timestep_ps * 1e-3 * 86400.0 / seconds_per_step


def workload(name: str, seed: int):
    from rainmd_b200 import synthetic
    from rainmd_b200.topology import build_system

    if name == "water-23558":
        topo, pos = synthetic.water_box(23558, seed=seed)
    elif name == "water-2854":
        topo, pos = synthetic.water_box(2854, seed=seed)
    elif name == "water-99999":
        topo, pos = synthetic.water_box(99999, seed=seed)
    elif name == "chain-1190":
        topo, pos = synthetic.config0(seed=seed)
    else:
        raise SystemExit(f"unknown workload {name}")
    system = build_system(topo, cutoff=0.9)
    box = system["boxVectors"]
    grid = [smooth_at_least(math.ceil(box[4 * d] / 0.1)) for d in range(3)]
    return system, pos, grid


def smooth_at_least(n: int) -> int:
    while True:
        r = n
        for p in (2, 3, 5):
            while r % p == 0:
                r //= p
        if r == 1:
            return n
        n += 1


# Neighbour-list skin (nm). 0.25 nm for the water boxes: on the 23,558-atom NPT box a sweep of
# 0.10 / 0.15 / 0.20 / 0.25 / 0.30 nm gave 0.118 / 0.115 / 0.112 / 0.111 / 0.111 ms a step (fewer
# rebuilds against longer rows); --skin overrides it. The small boxes of config 0 and the batch
# (2.3-4.9 nm) keep 0.15 nm, below the 0.9 (L/2 - rc) cap of the reference's skinFor
# (cells.js:67-91) on the smallest of them.
LIST_SKIN = 0.25
SMALL_BOX_SKIN = 0.15


def options_for(grid, seed, skin=None):
    return {"timestep": TIMESTEP_PS, "temperature": 300.0, "friction": 1.0, "seed": seed,
            "pmeOrder": 4, "grid": grid, "ewaldTolerance": 5e-4, "waterSolver": 1,
            "skin": LIST_SKIN if skin is None else skin, "rebuildInterval": 10, "adaptiveRebuild": True,
            "dispersionCorrection": True}


def batch_workload(seed: int = 0, count: int = 64):
    """64 solvated random-walk chains (20-400 chain atoms), totals log-uniform in 1,000-12,000
    atoms, each with its own PME grid at <= 1 A spacing."""
    from rainmd_b200 import synthetic
    from rainmd_b200.topology import build_system

    out = []
    for topo, pos in synthetic.batch(count, seed=seed):
        system = build_system(topo, cutoff=0.9)
        box = system["boxVectors"]
        grid = [smooth_at_least(math.ceil(box[4 * d] / 0.1)) for d in range(3)]
        out.append((system, pos, grid))
    return out


def batched_block(steps: int, seed: int, single_steps: int = 200, rank: int = 0, world: int = 1,
                  reduce_max=None):
    """Batched aggregate ns/day of the 64 uneven systems advanced together (one set of launches
    per step, CUDA-graph blocks of 100 steps): the sum over systems of each one's ns/day in the
    batch. Beside it the plain path for the same work: the same systems run one after another
    on the same GPU, each alone (aggregate = systems x ns/day at the summed per-system step
    time), and the ratio of the two, which is the summed single-system step time over the
    batch's step time. On N GPUs the systems are partitioned whole across the ranks
    (rainmd_b200.partition: no per-step collective); each rank advances its share as one batch,
    and the slowest rank's step time sets both figures."""
    from rainmd_b200.partition import partition_systems, system_cost
    from rainmd_b200.simulation import BatchSimulation, GpuSimulation

    def slowest(x):
        return reduce_max(x) if reduce_max is not None and world > 1 else x

    items = batch_workload(seed)
    systems = [s for s, _, _ in items]
    options = [options_for(g, seed=11 + k, skin=SMALL_BOX_SKIN) for k, (_, _, g) in enumerate(items)]
    atoms = [s["topology"]["atomCount"] for s in systems]
    costs = [system_cost(a, float(np.prod(np.asarray(s["boxVectors"], dtype=np.float64)[[0, 4, 8]])), 0.9, g)
             for a, s, (_, _, g) in zip(atoms, systems, items)]
    parts = partition_systems(costs, world)
    mine = parts[rank]
    ms_per_step, single_ms, shapes = 0.0, [], None
    if mine:
        batch = BatchSimulation([systems[k] for k in mine], [options[k] for k in mine])
        for b, k in enumerate(mine):
            batch.setState(b, items[k][1])
        batch.initialise()
        batch.minimise(maxIterations=100, forceTolerance=1000.0)
        batch.run(500, blockSize=100)
        batch.benchRun(100, 100, flushL2=True)
        ms_per_step = batch.benchRun(steps, 100, flushL2=True) / steps
        shapes = batch.kernelShapes()
        batch.release()
        for k in mine:
            sim = GpuSimulation(systems[k], options[k])
            sim.setState(items[k][1])
            sim.initialise()
            sim.minimise(maxIterations=100, forceTolerance=1000.0)
            sim.run(200, blockSize=100)
            single_ms.append(sim.benchRun(single_steps, 100, flushL2=True) / single_steps)
            sim.release()
    batch_ms = slowest(ms_per_step)
    sequential_ms = slowest(float(sum(single_ms)))
    batch_ns = len(systems) * ns_per_day(batch_ms * 1e-3)
    sequential_ns = len(systems) * ns_per_day(sequential_ms * 1e-3)
    loads = [sum(costs[k] for k in p) for p in parts]
    out = {"systems": len(systems), "atoms_total": int(sum(atoms)), "atoms_min": int(min(atoms)),
           "atoms_max": int(max(atoms)), "steps": steps, "ms_per_step": batch_ms,
           "aggregate_ns_per_day": batch_ns,
           "sequential_single_ms_per_step_summed": sequential_ms,
           "sequential_single_aggregate_ns_per_day": sequential_ns,
           "ratio_vs_sequential_singles": batch_ns / sequential_ns,
           "single_steps": single_steps, "seed": seed,
           "partition": {"ranks": world, "systems_per_rank": [len(p) for p in parts],
                         "cost_max_over_mean": max(loads) / (sum(loads) / world)}}
    if world == 1:
        out["single_ns_per_day_min"] = ns_per_day(max(single_ms) * 1e-3)
        out["single_ns_per_day_max"] = ns_per_day(min(single_ms) * 1e-3)
    if shapes is not None:
        out["kernel_shapes"] = {k: shapes[k] for k in ("neighbourGroupAtoms", "nonbondedLanes", "spreadAtomsPerBlock")}
    return out


def blocking_se(series):
    """Standard error of the mean of a correlated series by blocking (Flyvbjerg and Petersen,
    J. Chem. Phys. 91, 461 (1989)): the series is halved into blocks of doubling length and the
    naive error of the block means is taken at each level; the largest value over the levels
    that keep at least 8 blocks is returned, so correlations shorter than the blocks are
    counted."""
    x = np.asarray(series, dtype=np.float64)
    best = x.std(ddof=1) / math.sqrt(len(x)) if len(x) > 1 else 0.0
    while len(x) >= 16:
        x = 0.5 * (x[: len(x) // 2 * 2: 2] + x[1: len(x) // 2 * 2: 2])
        best = max(best, x.std(ddof=1) / math.sqrt(len(x)))
    return float(best)


def learned_barostat_study(ps: float, seeds=(3, 4, 5), warmup_moves: int = 2000):
    """23,558 atoms (a 300-atom chain and TIP3P water) started underdense at 0.60 g/cm^3, NPT
    at 1 bar and 300 K with a volume move every 25 steps, run as pairs from the same start: the
    plain exact barostat and the learned one (pre-trained on the first `warmup_moves` exact
    moves, then screening and training online), one pair per seed. Density and isothermal
    compressibility from the moves after the learned arm's warm-up (the final four fifths of
    each run; the density trajectory by tenths shows the relaxation from the underdense start),
    with the blocking-analysis standard error of each arm's mean density; per pair and pooled
    over the pairs, the learned-minus-plain density difference in units of its combined
    standard error; exact evaluations and wall time."""
    from rainmd_b200 import synthetic
    from rainmd_b200.simulation import GpuSimulation
    from rainmd_b200.topology import build_system

    steps = int(round(ps / TIMESTEP_PS))
    moves = steps // 25
    kT = 0.0083144626 * 300.0
    out = {"study": "learned-barostat", "ps": ps, "moves": moves, "warmup_moves": warmup_moves,
           "seeds": list(seeds), "pairs": []}
    for seed in seeds:
        topo, pos = synthetic.solvated_chain(23558, 300, density=0.60, seed=seed)
        system = build_system(topo, cutoff=0.9)
        box = system["boxVectors"]
        grid = [smooth_at_least(math.ceil(box[4 * d] / 0.1)) for d in range(3)]
        mass = float(np.sum(system["topology"]["masses"]))
        pair = {"seed": seed, "atoms": system["topology"]["atomCount"], "grid": grid, "start_density_g_cm3": 0.60}
        for learned in (False, True):
            options = options_for(grid, seed=seed)
            options.update({"pressure": 1.0, "barostatInterval": 25, "learnedBarostat": 1 if learned else 0,
                            "learnedWarmupMoves": warmup_moves})
            sim = GpuSimulation(system, options)
            sim.setState(pos)
            sim.initialise()
            sim.minimise(maxIterations=200, forceTolerance=1000.0)
            volumes = []
            t0 = time.perf_counter()
            for _ in range(moves):
                sim.run(25)
                volumes.append(sim.diagnostics()["volume"])
            wall = time.perf_counter() - t0
            trajectory = mass / np.array(volumes) * 1.66053906660e-3  # g/cm^3 per move
            v = np.array(volumes[len(volumes) // 5:])
            density = mass / v * 1.66053906660e-3
            d = sim.diagnostics()
            arm = {"density_by_tenth_of_run": [round(float(x.mean()), 4) for x in np.array_split(trajectory, 10)],
                   "density_g_cm3": float(density.mean()),
                   "density_se": blocking_se(density),
                   # kappa_T = <dV^2> / (kT <V>): nm^3 / (kJ/mol) -> 1/bar is x 6.0221e-2
                   "compressibility_per_bar": float(v.var() / (kT * v.mean()) * 6.02214076e-2),
                   "attempts": d["barostat_attempts"], "accepted": d["barostat_accepted"],
                   "exact_evaluations": d["barostat_exact_evaluations"], "screened": d["barostat_screened"],
                   "window_nm3": d["volume_scale"], "wall_s": wall,
                   "ns_per_day_wall": ns_per_day(wall / (moves * 25))}
            if learned:
                r = sim.surrogateReport()
                after = max(1, r["attempts"] - warmup_moves)
                arm.update({"surrogate_prediction_error_kT": r["prediction_error_kT"],
                            "surrogate_train_steps": r["train_steps"],
                            "exact_saved_after_warmup": 1.0 - (r["exact_evaluations"] - warmup_moves) / after,
                            "exact_saved_overall": 1.0 - r["exact_evaluations"] / max(1, r["attempts"])})
            pair["learned" if learned else "plain"] = arm
            sim.release()
        p, l = pair["plain"], pair["learned"]
        pair["difference_g_cm3"] = l["density_g_cm3"] - p["density_g_cm3"]
        pair["difference_se"] = math.hypot(p["density_se"], l["density_se"])
        pair["difference_sigma"] = pair["difference_g_cm3"] / pair["difference_se"]
        out["pairs"].append(pair)
    count = len(out["pairs"])
    diff = sum(pp["difference_g_cm3"] for pp in out["pairs"]) / count
    se = math.sqrt(sum(pp["difference_se"] ** 2 for pp in out["pairs"])) / count
    out["pooled_difference_g_cm3"] = diff
    out["pooled_difference_se"] = se
    out["pooled_difference_sigma"] = diff / se
    out["exact_saved_after_warmup_mean"] = float(np.mean([pp["learned"]["exact_saved_after_warmup"]
                                                           for pp in out["pairs"]]))
    return out


def trajectory_study(frames: int = 50, seed: int = 2):
    """Trajectory output from the device (shared/traj/*.js restated in csrc/traj.cu): per
    DCD frame and per restart, the whole call through the public API (imaging and packing
    on the device, one copy of the finished bytes to the host), next to the position read
    alone that any host-side writer starts from, and the CPU restatement of the writer."""
    import oracle.traj as ot
    from rainmd_b200 import traj
    from rainmd_b200.simulation import GpuSimulation

    out = {"study": "trajectory"}
    for name in ("water-23558", "water-99999"):
        system, pos, grid = workload(name, seed)
        n = system["topology"]["atomCount"]
        sim = GpuSimulation(system, options_for(grid, seed))
        sim.setState(pos)
        sim.initialise()
        sim.minimise(maxIterations=20, forceTolerance=1000.0)
        sim.run(500, blockSize=100)
        writer = traj.DcdWriter(n, TIMESTEP_PS, 1, periodic=True)
        writer.appendFrame(sim)
        t0 = time.perf_counter()
        for _ in range(frames):
            writer.appendFrame(sim)
        dcd_ms = (time.perf_counter() - t0) * 1e3 / frames
        traj.writeRestart(sim)
        t0 = time.perf_counter()
        for _ in range(10):
            text = traj.writeRestart(sim)
        rst7_ms = (time.perf_counter() - t0) * 1e3 / 10
        t0 = time.perf_counter()
        for _ in range(frames):
            state = sim.readState()
        read_ms = (time.perf_counter() - t0) * 1e3 / frames
        t = system["topology"]
        t0 = time.perf_counter()
        ot.dcd_frame(state["positions"].astype(np.float64), state["boxVectors"], t["moleculeOfAtom"],
                     t["moleculeCount"])
        cpu_dcd_ms = (time.perf_counter() - t0) * 1e3
        frame_bytes = len(writer.chunks[0])
        out[name] = {"atoms": n, "dcd_frame_bytes": frame_bytes, "dcd_ms_per_frame": dcd_ms,
                     "dcd_frame_gb_per_s": frame_bytes / (dcd_ms * 1e-3) / 1e9,
                     "restart_bytes": len(text), "restart_ms": rst7_ms,
                     "read_state_ms": read_ms,
                     "cpu_oracle_dcd_ms_per_frame": cpu_dcd_ms}
        sim.release()
    return out


def render_study(frames: int = 20, seed: int = 2):
    """The headless viewer (csrc/raster.cu): a 1920x1080 frame of every atom of the
    23,558-atom box as sphere impostors, through the public API (styles and camera in, the
    RGBA image out), next to the CPU restatement of the same frame."""
    import oracle
    from rainmd_b200.simulation import GpuSimulation
    from rainmd_b200.viewer import StructureViewer

    system, pos, grid = workload("water-23558", seed)
    t = system["topology"]
    t = dict(t)
    t.setdefault("atomicNumbers", [8 if m > 10 else 1 for m in t["masses"]])
    sim = GpuSimulation(system, options_for(grid, seed))
    sim.setState(pos)
    viewer = StructureViewer(1920, 1080)
    viewer.setStructure(t, positions=pos)
    viewer.draw(sim)
    t0 = time.perf_counter()
    for _ in range(frames):
        image = viewer.draw(sim)
    ms = (time.perf_counter() - t0) * 1e3 / frames
    t0 = time.perf_counter()
    expected = oracle.render(sim.readState()["positions"], viewer.camera(), viewer.styles, width=1920,
                             height=1080)
    cpu_ms = (time.perf_counter() - t0) * 1e3
    return {"study": "render", "atoms": t["atomCount"], "width": 1920, "height": 1080,
            "ms_per_frame": ms, "frames_per_s": 1e3 / ms, "cpu_oracle_ms_per_frame": cpu_ms,
            "identical_to_oracle": bool(np.array_equal(image, expected)),
            "covered_pixels": int((image[..., :3] != image[0, 0, :3]).any(-1).sum())}


def large_combined_study(steps: int, seed: int = 5):
    """250,000 atoms (a 4,000-atom chain in TIP3P water, PME order 4 on 128^3) advanced in one
    batch with 16 solvated systems of 5,000-20,000 atoms, all NPT at 1 bar with the learned
    barostat. Reports ns/day, each kernel group's algorithmic HBM bytes per launch over its
    CUDA-event time against the measured peak, and the large system's energy terms against
    the FP64 oracle at the positions and box the run ends with."""
    import oracle
    from rainmd_b200 import synthetic
    from rainmd_b200.simulation import BatchSimulation
    from rainmd_b200.topology import build_system

    rng = np.random.default_rng(seed)
    topo, pos = synthetic.solvated_chain(250000, 4000, seed=seed)
    items = [(build_system(topo, cutoff=0.9), pos, [128, 128, 128])]
    for k, size in enumerate(np.exp(rng.uniform(math.log(5000), math.log(20000), size=16)).astype(int)):
        t, p = synthetic.solvated_chain(int(size), int(rng.integers(20, 401)), seed=seed * 100 + k)
        system = build_system(t, cutoff=0.9)
        box = system["boxVectors"]
        items.append((system, p, [smooth_at_least(math.ceil(box[4 * d] / 0.1)) for d in range(3)]))
    systems = [s for s, _, _ in items]
    options = []
    for k, (_, _, grid) in enumerate(items):
        o = options_for(grid, seed=seed + k)
        o.update({"pressure": 1.0, "barostatInterval": 25, "learnedBarostat": 1, "learnedWarmupMoves": 200})
        options.append(o)
    batch = BatchSimulation(systems, options)
    for k, (_, p, _) in enumerate(items):
        batch.setState(k, p)
    batch.initialise()
    batch.minimise(maxIterations=100, forceTolerance=1000.0)
    batch.run(1000, blockSize=100)
    batch.benchRun(100, 100, flushL2=True)
    ms = batch.benchRun(steps, 100, flushL2=True)
    atoms = [s["topology"]["atomCount"] for s in systems]
    n = sum(atoms)
    per_step_ns = ns_per_day(ms * 1e-3 / steps)
    peak, peak_kind = measured_peaks()
    # algorithmic bytes per launch over the whole batch (the same formulas as the main line;
    # P from the neighbour estimate rho 4/3 pi rc^3 / 2 per atom)
    pairs = sum(a * (a / float(s["boxVectors"][0] * s["boxVectors"][4] * s["boxVectors"][8])) *
                (4.0 / 3.0) * math.pi * 0.9 ** 3 / 2 for a, s in zip(atoms, systems))
    k3 = sum(g[0] * g[1] * g[2] for _, _, g in items)
    half = sum(g[0] * g[1] * (g[2] // 2 + 1) for _, _, g in items)
    kernels = {}
    for name, nbytes in (("nonbonded", 20 * n + 4 * pairs + 24 * n), ("pme", 32 * n + 24 * n + 16 * k3 + 32 * half),
                         ("integrate", (52 + 24) * n)):
        t = batch.timeKernel(name, reps=20)
        kernels[name] = {"ms": t, "gb_per_s": nbytes / (t * 1e-3) / 1e9, "frac_of_peak": nbytes / (t * 1e-3) / 1e9 / peak}
    # the large system against the FP64 oracle, at the run's final positions and box
    state = batch.readState(0)
    held = state["positions"].astype(np.float64)
    energy, _ = batch.debugEvaluate(0)
    ref_system = dict(systems[0])
    ref_system["boxVectors"] = np.array(state["boxVectors"], dtype=np.float64)
    alpha = math.sqrt(-math.log(2.0 * 5e-4)) / 0.9
    expect, _ = oracle.Oracle(ref_system).potential(held, method="PME", alpha=alpha, grid=[128, 128, 128], order=4)
    errors = {
        "lennardJones": abs(energy["lennard_jones"] - expect["lennardJones"]) / abs(expect["lennardJones"]),
        "coulombDirect": abs(energy["coulomb_direct"] - expect["coulombDirect"]) / abs(expect["coulombDirect"]),
        "coulombReciprocal": abs(energy["coulomb_reciprocal"] - expect["coulombReciprocal"]) / abs(expect["coulombReciprocal"]),
        "bonded": abs(energy["bonded"] - expect["bonded"]) / abs(expect["bonded"]),
        "potential_without_dispersion": abs(energy["potential"] - energy["dispersion"] - expect["total"]) / abs(expect["total"]),
    }
    reports = [batch.surrogateReport(k) for k in range(len(systems))]
    out = {"study": "large-combined", "systems": len(systems), "atoms_large": atoms[0], "atoms_total": n,
           "small_atoms": atoms[1:], "steps": steps, "ms_per_step": ms / steps,
           "large_ns_per_day": per_step_ns, "aggregate_ns_per_day": per_step_ns * len(systems),
           "kernels": kernels, "peak_gb_per_s": peak, "peak_source": peak_kind,
           "large_energy_relative_error_vs_fp64_oracle": errors,
           "barostat": {"attempts": int(sum(r["attempts"] for r in reports)),
                        "exact_evaluations": int(sum(r["exact_evaluations"] for r in reports)),
                        "screened": int(sum(r["screened"] for r in reports)),
                        "exact_passes": reports[0]["exact_passes"], "skipped_passes": reports[0]["skipped_passes"]},
           "kernel_shapes": {k: v for k, v in batch.kernelShapes().items() if k != "tuned"},
           "seed": seed}
    batch.release()
    return out


def measured_traffic(kernel: str, workload_name: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary of this workload
    (profiles/<kernel>_<workload>.md, line 'dram_bytes_per_launch: N'), else None."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload_name}.md")
    try:
        with open(path) as handle:
            for line in handle:
                if line.strip().startswith("dram_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        return None
    return None


def unique_pairs_within(positions, box_length, cutoff):
    from scipy.spatial import cKDTree

    p = np.mod(positions.reshape(-1, 3), box_length)
    tree = cKDTree(p, boxsize=box_length)
    return len(tree.query_pairs(cutoff, output_type="ndarray"))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device = device_index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        try:
            with open(self.file.name) as handle:
                rows = [line.strip().split(", ") for line in handle if line.strip()]
        except OSError:
            rows = []
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4)
                          if len(r) > 5 + k and r[5 + k].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# The pair kernel's arithmetic ceiling, reported beside its memory roofline. The group-pair
# kernel evaluates every pair within the cutoff once (the per-atom-row kernel twice, once from
# each atom), and one evaluation of the force-only precision form issues, counted from the
# kernels' source: 49 FP32 operations (47 in the group-pair kernel, which folds the fixed-point
# scale into the force's scalar factor once instead of scaling each component), 6 integer
# operations (three 64-bit fixed-point adds), 3 SFU operations (rsqrt, ex2, rcp) and 3
# float-to-int64 conversions. The ceiling is the larger
# of the issue time (one instruction per lane per clock, 128 lanes per SM) and the
# SFU-and-conversion time (16 lanes per SM per clock) on 148 SMs at the SM clock sampled during
# the run. List walking, loads, out-of-cutoff entries, the partner's reduction and atomics and
# the exception loop are not counted, so the kernel cannot reach it.
PAIR_XU_OPS = 3 + 3
B200_SMS = 148


def pair_arithmetic_ceiling(pairs, kernel_ms, sm_mhz, evaluations_per_pair=1):
    evaluations = evaluations_per_pair * int(pairs)
    lane_ops = (47 if evaluations_per_pair == 1 else 49) + 6 + 3 + 3
    clock = float(sm_mhz) * 1e6
    issue_s = evaluations * lane_ops / (B200_SMS * 128 * clock)
    xu_s = evaluations * PAIR_XU_OPS / (B200_SMS * 16 * clock)
    ceiling_ms = max(issue_s, xu_s) * 1e3
    return {"evaluations": evaluations, "lane_ops_per_evaluation": lane_ops,
            "sfu_and_conversion_ops_per_evaluation": PAIR_XU_OPS, "sm_mhz": float(sm_mhz),
            "ceiling_ms": ceiling_ms, "frac": ceiling_ms / kernel_ms}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as handle:
            data = json.load(handle)
        return float(data["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_baseline(system, positions, grid, seed, budget_s=20.0, threads=None, npt=False):
    """The reference's CPU path on the host cores for a bounded sample of the workload: the
    oracle's runDynamics (cpu/simulation.js:114-156 restated, FP64, O(N^2) direct space,
    naive-DFT PME) for a few steps and, for an NPT workload, one volume move of the oracle's
    attemptVolumeChange restatement (webgpu/simulation.js:995-1070; the reference's CPU path
    has no barostat of its own), amortised at one move every 25 steps."""
    import oracle

    threads = threads or (os.cpu_count() or 1)
    oracle.set_threads(threads)
    o = oracle.Oracle(system)
    alpha = oracle.alpha_from_tolerance(0.9, 5e-4)
    integ = o.integrator(timestep=TIMESTEP_PS, temperature=300.0, friction=1.0, seed=seed, tolerance=1e-5)
    vel = np.zeros_like(positions)
    t0 = time.perf_counter()
    o.potential(positions, method="PME", alpha=alpha, grid=grid, order=4)
    per_eval = time.perf_counter() - t0
    steps = max(1, min(10, int(budget_s / max(per_eval, 1e-3))))
    t0 = time.perf_counter()
    pos1, vel1, _, _ = o.run_dynamics(positions, vel, steps, 0, integ, alpha, grid, 4)
    elapsed = time.perf_counter() - t0
    # run_dynamics evaluates the potential once before its loop
    per_step = max(1e-9, (elapsed - per_eval) / steps)
    sample = (f"{steps} BAOAB steps of the FP64 oracle (O(N^2) direct space, naive-DFT PME) on this "
              f"workload, {threads} thread{'s' if threads > 1 else ''}")
    if npt:
        box = system["boxVectors"]
        t0 = time.perf_counter()
        oracle.volume_move(system, pos1, vel1, 1, 0.01 * abs(box[0] * box[4] * box[8]), seed=seed,
                           temperature=300.0, pressure=1.0, alpha=alpha, grid=grid, order=4)
        move_s = time.perf_counter() - t0
        per_step += move_s / BAROSTAT_INTERVAL
        sample += f" and one volume move ({move_s:.2f} s) amortised over {BAROSTAT_INTERVAL} steps"
    oracle.set_threads(os.cpu_count() or 1)
    return {"value": ns_per_day(per_step), "unit": "ns/day", "cores": threads, "kind": "port",
            "sample": sample + f": {per_step * 1e3:.1f} ms/step", "ms_per_step": per_step * 1e3}


BAROSTAT_INTERVAL = 25


def run_reference(args, rank, world):
    if rank != 0:
        return
    system, pos, grid = workload(args.workload, seed=1)
    n = system["topology"]["atomCount"]
    npt = args.ensemble == "npt"
    base = cpu_baseline(system, pos, grid, seed=1, budget_s=args.reference_budget, npt=npt)
    line = {
        "impl": "reference", "metric": METRIC, "value": base["value"], "unit": "ns/day", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ns_to_ms(base["value"]),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)", "config": config_block(args, n, grid, world),
        "cpu_baseline": base,
        "e2e": {"value": base["value"], "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def aggregate(device_ms: float, steps: int, world: int, reduce_max=None):
    """Replica timing: the slowest rank's device time sets the time; every rank's
    simulated nanoseconds count. Returns (value ns/day, seconds per step)."""
    slowest = reduce_max(device_ms) if reduce_max is not None else device_ms
    seconds_per_step = slowest / 1e3 / steps
    return world * ns_per_day(seconds_per_step), seconds_per_step


def ns_to_ms(value_ns_day):
    return TIMESTEP_PS * 1e-3 * 86400.0 / value_ns_day * 1e3


def describe(name, grid, npt):
    what = {"water-23558": "TIP3P water", "water-2854": "TIP3P water", "water-99999": "TIP3P water",
            "chain-1190": "22-atom chain, Na+ and 389 TIP3P waters"}.get(name, name)
    ensemble = (f"NPT 1 bar (MC barostat, a move every {BAROSTAT_INTERVAL} steps)" if npt else "NVT")
    return (f"{name}: {what} {ensemble} 300 K, 2 fs, rc 0.9 nm, PME order 4 {grid[0]}x{grid[1]}x{grid[2]}, "
            f"SETTLE, Langevin 1/ps")


def config_block(args, atoms, grid, world):
    return {"workload": describe(args.workload, grid, args.ensemble == "npt"),
            "atoms": atoms, "replicas": world, "parallelism": f"replicas{world}",
            "l2": "flushed (256 MB written) before every timed block",
            "lists": "reference host schedule" if args.rebuild_schedule else "rebuilt on demand",
            "skin_nm": LIST_SKIN}


def prepare(system, pos, grid, seed, npt, args, skin=None):
    """A simulation of `system` minimised and equilibrated (untimed), with its block length:
    NPT runs in blocks of the barostat interval (a move at the start of each block, as the
    reference's run() attempts one at block boundaries), NVT in blocks of 100 steps."""
    from rainmd_b200.simulation import GpuSimulation

    opts = options_for(grid, seed=seed, skin=skin)
    if args.pair_list is not None:
        opts["pairList"] = args.pair_list
    if args.nonbonded_lanes is not None:
        opts["nonbondedLanes"] = args.nonbonded_lanes
    if npt:
        opts.update({"pressure": 1.0, "barostatInterval": BAROSTAT_INTERVAL})
    if args.rebuild_schedule:
        opts["rebuildOnDemand"] = False
    sim = GpuSimulation(system, opts)
    sim.setState(pos)
    sim.initialise()
    sim.minimise(maxIterations=args.minimise, forceTolerance=1000.0)
    block = BAROSTAT_INTERVAL if npt else args.block
    sim.run(args.equilibrate, blockSize=block)
    return sim, block


def timed(sim, steps, warmup, block, barrier, min_warm_s=0.0):
    """W warm-up blocks of `block` steps (and more until `min_warm_s` of wall time has passed, so
    a clock sampler started before them sees the GPU under load), then exactly `steps` steps
    timed with CUDA events on the engine's stream in blocks of at most `block`, L2 flushed
    before every block. With the barostat, a block is the move interval: a move is due when the
    timed region starts, and it holds one move per started interval (at 20 steps, one move).
    Returns device ms and the kernels launched, lists built and volume moves attempted inside
    the timed region."""
    t0 = time.perf_counter()
    done = 0
    while done < max(3, warmup) or time.perf_counter() - t0 < min_warm_s:
        sim.benchRun(block, block, flushL2=True)
        done += 1
    launches0 = sim.kernelLaunches()
    builds0 = sim.diagnostics()["list_builds"]
    moves0 = sim.diagnostics()["barostat_attempts"]
    barrier()
    device_ms = sim.benchRun(steps, min(block, steps), flushL2=True)
    barrier()
    d = sim.diagnostics()
    return device_ms, sim.kernelLaunches() - launches0, d["list_builds"] - builds0, d["barostat_attempts"] - moves0


def end_to_end(sim, n, steps, block, barrier, npt):
    """The same steps through the public API with host arrays: setState (host f64 positions and
    velocities), initialise, run, readState (host f32). With the barostat, an untimed block of
    one move interval first, so that a move is due when the timed call starts, as in the
    device-timed region. Returns (seconds, h2d bytes, d2h bytes, final state)."""
    if npt:
        sim.run(BAROSTAT_INTERVAL, blockSize=BAROSTAT_INTERVAL)
    state = sim.readState()
    host_pos = state["positions"].astype(np.float64)
    host_vel = state["velocities"].astype(np.float64)
    # one untimed pass of the same calls first: the step graph that a fresh state starts with
    # (its first step rebuilds the lists unconditionally) is captured once, as a user's second
    # and later calls find it
    sim.setState(host_pos, host_vel, step=sim.step)
    sim.initialise()
    sim.run(steps, blockSize=min(block, steps))
    sim.readState()
    if npt:
        sim.run(BAROSTAT_INTERVAL, blockSize=BAROSTAT_INTERVAL)
    state = sim.readState()
    host_pos = state["positions"].astype(np.float64)
    host_vel = state["velocities"].astype(np.float64)
    barrier()
    t0 = time.perf_counter()
    sim.setState(host_pos, host_vel, step=sim.step)
    sim.initialise()
    sim.run(steps, blockSize=min(block, steps))
    out = sim.readState()
    seconds = time.perf_counter() - t0
    assert np.all(np.isfinite(out["positions"]))
    return seconds, 2 * 16 * n, (16 + 16 + 24) * n + 8 * 9, out


def config0_line(args, barrier):
    """The reference's published configuration: 1,190 atoms (a 22-atom chain, Na+ and 389 TIP3P
    waters in a 2.265 nm box), NPT at 1 bar with a move every 25 steps, PME order 4 on 24^3 —
    device-timed, end to end through the API, and the CPU path single-threaded and on all
    cores. The reference reports 133 ns/day for this system on Apple M-series WebGPU."""
    system, pos, grid = workload("chain-1190", seed=1)
    n = system["topology"]["atomCount"]
    sim, block = prepare(system, pos, grid, seed=7, npt=True, args=args, skin=SMALL_BOX_SKIN)
    steps = max(args.steps, 100)
    device_ms, launches, builds, moves = timed(sim, steps, args.warmup, block, barrier)
    seconds, h2d, d2h, _ = end_to_end(sim, n, steps, block, barrier, True)
    out = {"workload": describe("chain-1190", grid, True), "atoms": n, "steps": steps,
           "ms_per_step": device_ms / steps, "value": ns_per_day(device_ms * 1e-3 / steps), "unit": "ns/day",
           "volume_moves_timed": moves, "list_builds_timed": builds, "gpu_launches": launches,
           "e2e": {"value": ns_per_day(seconds / steps), "unit": "ns/day", "h2d_bytes_per_step": h2d / steps,
                   "d2h_bytes_per_step": d2h / steps},
           "reference_published": {"value": 133, "unit": "ns/day",
                                   "where": "Apple M-series WebGPU (the reference's docs/STATUS.md:184)"}}
    sim.release()
    if not args.no_cpu_baseline:
        out["cpu_baseline_single_thread"] = cpu_baseline(system, pos, grid, seed=1, budget_s=5.0, threads=1,
                                                         npt=True)
        out["cpu_baseline_all_cores"] = cpu_baseline(system, pos, grid, seed=1, budget_s=5.0, npt=True)
    return out


def main():
    global LIST_SKIN
    parser = argparse.ArgumentParser()
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=2000)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", default="ours", choices=["ours", "reference"])
    parser.add_argument("--workload", default="water-23558")
    parser.add_argument("--ensemble", default="npt", choices=["npt", "nvt"],
                        help="NPT (the default): 1 bar, a Monte Carlo volume move every 25 steps")
    parser.add_argument("--block", type=int, default=100, help="steps per graph block in NVT")
    parser.add_argument("--reference-budget", type=float, default=20.0)
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--minimise", type=int, default=200, help="minimiser iterations before dynamics")
    parser.add_argument("--equilibrate", type=int, default=3000, help="untimed steps before warm-up")
    parser.add_argument("--no-batched", action="store_true", help="skip the 64-system batch measurement")
    parser.add_argument("--no-extra", action="store_true",
                        help="skip the NVT comparison and the 1,190-atom configuration")
    parser.add_argument("--study", choices=["learned-barostat", "large-combined", "trajectory", "render"],
                        default=None,
                        help="run a study instead of the benchmark and print its JSON line")
    parser.add_argument("--ps", type=float, default=500.0, help="length of a study run")
    parser.add_argument("--seeds", type=int, nargs="+", default=[3, 4, 5],
                        help="seeds of the learned-barostat study's pairs of runs")
    parser.add_argument("--batch-steps", type=int, default=500)
    parser.add_argument("--pair-list", type=int, choices=[0, 1], default=None,
                        help="neighbour structure of the pair loop: 0 group-pair rows, 1 per-atom rows "
                             "(default: the engine's)")
    parser.add_argument("--skin", type=float, default=None,
                        help=f"neighbour-list skin in nm (default {LIST_SKIN})")
    parser.add_argument("--nonbonded-lanes", type=int, choices=[32, 64, 128], default=None,
                        help="fix the group-pair kernel's lanes a row instead of autotuning them")
    parser.add_argument("--rebuild-schedule", action="store_true",
                        help="rebuild the lists on the reference's host schedule instead of on demand "
                             "(the same kernels; ncu profiles no kernel of a graph with conditional nodes)")
    args = parser.parse_args()
    if args.skin is not None:
        LIST_SKIN = float(args.skin)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.study is not None:
        if rank == 0:
            studies = {"learned-barostat": lambda: learned_barostat_study(args.ps, seeds=tuple(args.seeds)),
                       "large-combined": lambda: large_combined_study(args.steps),
                       "trajectory": trajectory_study, "render": render_study}
            # the clock record covers the whole study (nvidia-smi every 200 ms)
            with ClockSampler(local) as clocks:
                result = studies[args.study]()
            summary = clocks.summary()
            summary["window"] = "the whole study"
            result["clocks"] = summary
            print(json.dumps(result), flush=True)
        return
    # one GPU per process: make this rank's GPU device 0 before any CUDA initialisation
    if world > 1:
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local)
    import torch
    import torch.distributed as dist

    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        torch.cuda.set_device(0)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def reduce_max(x):
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    npt = args.ensemble == "npt"
    system, pos, grid = workload(args.workload, seed=1 + rank)
    n = system["topology"]["atomCount"]
    sim, block = prepare(system, pos, grid, seed=7 + rank, npt=npt, args=args)
    with ClockSampler(local if world == 1 else 0) as clocks:
        device_ms, launches, builds, moves = timed(sim, args.steps, args.warmup, block, barrier, min_warm_s=1.5)
    value, seconds_per_step = aggregate(device_ms, args.steps, world, reduce_max)

    # energies stay finite and the run was physical
    diag = sim.diagnostics()
    e = sim.energy()

    # end to end through the public API: host arrays in, run, host arrays out
    e2e_seconds, h2d, d2h, out = end_to_end(sim, n, args.steps, block, barrier, npt)
    e2e_value = world * ns_per_day(reduce_max(e2e_seconds) / args.steps)

    # roofline of the dominant kernel (nonbonded): algorithmic bytes per launch over the
    # CUDA-event launch time on the engine's stream
    pairs = unique_pairs_within(out["positions"].astype(np.float64), out["boxVectors"][0], 0.9)
    nb_ms = sim.timeKernel("nonbonded", reps=50)
    shapes = sim.kernelShapes()
    pair_list = sim.diagnostics()["pair_list"]
    pme_ms = sim.timeKernel("pme", reps=50)
    integ_ms = sim.timeKernel("integrate", reps=50)
    rebuild_ms = sim.timeKernel("rebuild", reps=20)
    bytes_nb = 20 * n + 4 * pairs + 24 * n
    h = grid[0] * grid[1] * (grid[2] // 2 + 1)
    k3 = grid[0] * grid[1] * grid[2]
    bytes_pme = 32 * n + 24 * n + 16 * k3 + 32 * h
    peak, peak_kind = measured_peaks()
    achieved = bytes_nb / (nb_ms * 1e-3) / 1e9
    sim.release()
    # the reference's per-atom rows on the same positions: their pair kernel (each pair from both
    # atoms; the autotuned lanes, and the per-lane f32 form) and their search
    from rainmd_b200.simulation import GpuSimulation
    rows = GpuSimulation(system, dict(options_for(grid, seed=7 + rank), pairList=1))
    rows.setState(out["positions"].astype(np.float64), out["velocities"].astype(np.float64))
    rows.initialise()
    atom_rows = {"nonbonded": rows.timeKernel("nonbonded", reps=50), "rebuild_kernels": rows.timeKernel("rebuild", reps=20),
                 "kernel_shapes": {k: rows.kernelShapes()[k] for k in ("neighbourGroupAtoms", "nonbondedLanes")}}
    rows.setNonbonded(atom_rows["kernel_shapes"]["nonbondedLanes"], pairFixed=False)
    atom_rows["nonbonded_per_lane_f32"] = rows.timeKernel("nonbonded", reps=50)
    rows.release()

    extra = {}
    if not args.no_extra:
        # the same box without the barostat (the precision study's NVT form)
        other = "nvt" if npt else "npt"
        sim2, block2 = prepare(system, pos, grid, seed=7 + rank, npt=not npt, args=args)
        ms2, launches2, builds2, moves2 = timed(sim2, args.steps, args.warmup, block2, barrier)
        sim2.release()
        v2, sps2 = aggregate(ms2, args.steps, world, reduce_max)
        extra[other] = {"value": v2, "unit": "ns/day", "ms_per_step": sps2 * 1e3, "gpu_launches": launches2,
                        "list_builds_timed": builds2, "volume_moves_timed": moves2,
                        "workload": describe(args.workload, grid, not npt)}
        extra["config0"] = config0_line(args, barrier)
    batched = None if args.no_batched else batched_block(args.batch_steps, seed=0, rank=rank, world=world,
                                                          reduce_max=reduce_max)
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    base = None
    if not args.no_cpu_baseline:
        base = cpu_baseline(system, pos, grid, seed=1, npt=npt)
        base["single_thread"] = cpu_baseline(system, pos, grid, seed=1, budget_s=12.0, threads=1, npt=npt)
    traffic = measured_traffic("k_group_pairs" if pair_list != 1 else "k_nonbonded", args.workload)
    clock_summary = clocks.summary()
    clock_summary["window"] = "warm-up blocks (at least 1.5 s) and the timed region"
    sm_clock = clock_summary.get("sm_mhz") or clock_summary.get("sm_max_mhz") or 1965.0
    line = {
        "metric": METRIC, "value": value, "unit": "ns/day", "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": seconds_per_step * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": f"synthetic (seeded TIP3P lattice, minimised and equilibrated {args.equilibrate} steps)",
        "config": config_block(args, n, grid, world),
        "e2e": {"value": e2e_value, "unit": "ns/day", "h2d_bytes_per_step": h2d / args.steps,
                "d2h_bytes_per_step": d2h / args.steps,
                "path": "setState(host f64) + initialise + run(K) + readState(host f32)"},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": "k_group_pairs" if pair_list != 1 else "k_nonbonded",
                     "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                     "algorithmic_bytes": bytes_nb, "unique_pairs_within_cutoff": pairs,
                     "ms_per_launch": nb_ms,
                     "arithmetic_ceiling": pair_arithmetic_ceiling(pairs, nb_ms, sm_clock,
                                                                   1 if pair_list != 1 else 2)},
        "kernels_ms": {"nonbonded": nb_ms, "pme_kernels": pme_ms, "integrate": integ_ms,
                       "rebuild_kernels": rebuild_ms,
                       "pme_roofline_frac": bytes_pme / (pme_ms * 1e-3) / 1e9 / peak},
        "pair_list": {0: "group-pair rows", 1: "per-atom rows", 2: "group-pair rows (+ per-atom rows)"}[pair_list],
        "per_atom_rows_ms": atom_rows,
        "kernel_shapes": {k: shapes[k] for k in ("neighbourGroupAtoms", "nonbondedLanes", "spreadAtomsPerBlock")},
        "autotune_ms": shapes["tuned"],
        **extra,
        "batched": batched,
        "clocks": clock_summary,
        "physics": {"temperature": e["temperature"], "potential": e["potential"], "volume": e["volume"],
                    "list_builds_timed": builds, "steps_per_list_build": args.steps / max(builds, 1),
                    "volume_moves_timed": moves, "barostat_attempts": diag["barostat_attempts"],
                    "barostat_accepted": diag["barostat_accepted"],
                    "rebuild_on_demand": diag["rebuild_on_demand"],
                    "rebuild_interval": diag["rebuild_interval"], "skin_violations": diag["skin_violations"],
                    "neighbour_capacity": diag["neighbour_capacity"]},
        "cpu_baseline": base,
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
